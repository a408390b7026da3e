"""Plan 3 (phase A as plain sums over the precomputed digit table) against the
consensus vectors, the oracle and the other plans, for several window counts:
uniform windows (32 of 8 bits) and windows of two widths (29: 24 of 9 bits and
5 of 8; 26: 22 of 10 and 4 of 9; 24: 16 of 11 and 8 of 10; 23: 3 of 12 and 20
of 11)."""
import numpy as np
import pytest

import vkzg_b200
from conftest import adversarial_blobs, random_blobs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("windows", [32, 29, 26, 24, 23])
def test_plan3_mainnet_vectors(golden_proofs, monkeypatch, windows):
    """Every valid vector, batched, with the table's window count forced."""
    monkeypatch.delenv("VKZG_TABLES_PATH", raising=False)
    monkeypatch.delenv("VKZG_COMB_BITS", raising=False)
    monkeypatch.setenv("VKZG_PLAN", "3")
    monkeypatch.setenv("VKZG_COMB_WINDOWS", str(windows))
    n = len(golden_proofs["valid_names"])
    with vkzg_b200.Prover(max_batch_size=n) as p:
        out = p.compute_cell_kzg_proofs_batch(golden_proofs["valid_blobs"].tobytes(), n)
        d, _, nbytes = p.digit_table()
        assert d == windows and nbytes == vkzg_b200.comb_table_bytes(windows)
    for k in range(n):
        assert out[k * 6144:(k + 1) * 6144] == golden_proofs["valid_proofs"][k].tobytes(), k


def test_plan3_synthetic_vs_oracle(synthetic, oracle, tmp_path, monkeypatch):
    """Seeded random and the four adversarial blobs under a synthetic setup,
    default window, against the oracle."""
    tau, mono, tables = synthetic
    path = str(tmp_path / "synthetic_tables.bin")
    vkzg_b200.write_tables(mono, path)
    monkeypatch.setenv("VKZG_TABLES_PATH", path)
    monkeypatch.setenv("VKZG_PLAN", "3")
    monkeypatch.delenv("VKZG_COMB_BITS", raising=False)
    monkeypatch.delenv("VKZG_COMB_WINDOWS", raising=False)
    blobs = np.concatenate([random_blobs(12, 303), adversarial_blobs()])
    out = np.zeros(len(blobs) * 6144, np.uint8)
    with vkzg_b200.Prover(max_batch_size=len(blobs)) as p:
        assert p.compute_proofs_raw(out, blobs, len(blobs)) == 0
        d, build_ms, nbytes = p.digit_table()
        # the default budget's candidates: 23 windows (3 of 12 bits, 20 of 11), the
        # most that fit, then 24 and 25 (an earlier tuner in the process may have
        # chosen one of them for these tables)
        assert d in (23, 24, 25) and nbytes == vkzg_b200.comb_table_bytes(d) <= 20 << 30
    rc, want = oracle.compute_proofs(tables, blobs)
    assert rc == 0
    for b in range(len(blobs)):
        assert np.array_equal(out[b * 6144:(b + 1) * 6144], want[b * 6144:(b + 1) * 6144]), b


def test_plans_agree_and_tuner_times_plan3(monkeypatch):
    """All plans give the same bytes at 32 blobs; a prover sized for 16 blobs or
    more times plan 3 at every size class (below 16 at one window count), a
    smaller prover never builds the table, and provers share one table."""
    monkeypatch.delenv("VKZG_TABLES_PATH", raising=False)
    monkeypatch.delenv("VKZG_PLAN", raising=False)
    monkeypatch.setenv("VKZG_COMB_BITS", "10")
    blobs = random_blobs(32, 404)
    outs = []
    for plan in range(vkzg_b200.PLANS):
        monkeypatch.setenv("VKZG_PLAN", str(plan))
        with vkzg_b200.Prover(max_batch_size=32) as p:
            out = np.zeros(32 * 6144, np.uint8)
            assert p.compute_proofs_raw(out, blobs, 32) == 0
            outs.append(out)
    for out in outs[1:]:
        assert np.array_equal(out, outs[0])
    monkeypatch.delenv("VKZG_PLAN")
    with vkzg_b200.Prover(max_batch_size=32) as p, vkzg_b200.Prover(max_batch_size=32) as q:
        table = p.autotune(32)
        assert table[32][1][3] > 0 and table[16][1][3] > 0 and table[8][1][3] > 0
        out = np.zeros(32 * 6144, np.uint8)
        assert p.compute_proofs_raw(out, blobs, 32) == 0
        assert np.array_equal(out, outs[0])
        q.autotune(16)
        assert q.digit_table()[1] == p.digit_table()[1]  # same table object: same build record
    with vkzg_b200.Prover(max_batch_size=8) as r:
        table = r.autotune(8)
        assert table[8][1][3] == -1 and r.digit_table() is None


def test_plan3_without_digit_table_falls_back(golden_proofs, monkeypatch):
    """With the digit table disabled ($VKZG_COMB_BITS=0, as when it cannot be
    allocated) a forced plan 3 runs as plan 4 and still proves the vectors."""
    monkeypatch.delenv("VKZG_TABLES_PATH", raising=False)
    monkeypatch.setenv("VKZG_PLAN", "3")
    monkeypatch.setenv("VKZG_COMB_BITS", "0")
    n = len(golden_proofs["valid_names"])
    with vkzg_b200.Prover(max_batch_size=n) as p:
        out = p.compute_cell_kzg_proofs_batch(golden_proofs["valid_blobs"].tobytes(), n)
        assert p.digit_table() is None
    assert out == golden_proofs["valid_proofs"].tobytes()


def test_tuner_times_windows_within_budget(monkeypatch):
    """With a 12 GiB budget the tuner builds and times tables of 25, 26 and 27
    windows (the fewest whose table fits, 12.5 GB, and the next two counts),
    keeps the fastest, and reports each trial's table size; the proofs equal
    those of plan 0.  $VKZG_COMB_BITS, which pins the widest window, is unset."""
    monkeypatch.delenv("VKZG_TABLES_PATH", raising=False)
    monkeypatch.delenv("VKZG_PLAN", raising=False)
    monkeypatch.delenv("VKZG_COMB_BITS", raising=False)
    monkeypatch.delenv("VKZG_COMB_WINDOWS", raising=False)
    monkeypatch.setenv("VKZG_COMB_BUDGET_GB", "12")
    fits = [d for d in range(18, 33) if vkzg_b200.comb_table_bytes(d) <= 12 << 30][:3]
    assert fits == [25, 26, 27]
    blobs = random_blobs(32, 505)
    with vkzg_b200.Prover(max_batch_size=32) as p:
        table = p.autotune(32)  # largest size class first: the table is chosen at 32 blobs
        trials = p.window_trials(32)
        assert [t[0] for t in trials] == fits
        for d, nbytes, build_ms, ms in trials:
            assert nbytes == vkzg_b200.comb_table_bytes(d) and build_ms > 0 and ms > 0
        best = min(trials, key=lambda t: t[3])
        assert p.digit_table()[0] == best[0]
        assert abs(table[32][1][3] - best[3]) < 1e-9
        assert [t[0] for t in p.window_trials(16)] == [best[0]]  # smaller classes keep it
        out = np.zeros(32 * 6144, np.uint8)
        assert p.compute_proofs_raw(out, blobs, 32) == 0
        mem = p.device_bytes()
        assert mem["digit_table"] == vkzg_b200.comb_table_bytes(best[0]) <= 12 << 30
    monkeypatch.setenv("VKZG_PLAN", "0")
    with vkzg_b200.Prover(max_batch_size=32) as q:
        want = np.zeros(32 * 6144, np.uint8)
        assert q.compute_proofs_raw(want, blobs, 32) == 0
    assert np.array_equal(out, want)


def test_bits_alias_pins_the_widest_window(golden_proofs, monkeypatch):
    """$VKZG_COMB_BITS=c pins the table of ceil(256 / c) windows, whose widest
    window is c bits: 11 -> 24 windows (16 of 11 bits, 8 of 10)."""
    monkeypatch.delenv("VKZG_TABLES_PATH", raising=False)
    monkeypatch.delenv("VKZG_COMB_WINDOWS", raising=False)
    monkeypatch.setenv("VKZG_PLAN", "3")
    monkeypatch.setenv("VKZG_COMB_BITS", "11")
    assert max(vkzg_b200.comb_windows(24)) == 11
    blob = golden_proofs["valid_blobs"][1].tobytes()
    with vkzg_b200.Prover(max_batch_size=16) as p:
        out = p.compute_cell_kzg_proofs_batch(blob, 1)
        assert p.digit_table()[0] == 24
    assert out == golden_proofs["valid_proofs"][1].tobytes()


def test_default_prover_is_small(monkeypatch):
    """A prover with the default options batches 4 blobs per launch, as the
    reference's does, and holds well under 8 GB of device memory."""
    monkeypatch.delenv("VKZG_TABLES_PATH", raising=False)
    with vkzg_b200.Prover() as p:
        mem = p.device_bytes()
        assert mem["digit_table"] == 0
        assert mem["working"] + mem["tables"] < 1 << 30
        blobs = random_blobs(9, 606)  # three chunks of 4, 4 and 1
        out = np.zeros(9 * 6144, np.uint8)
        assert p.compute_proofs_raw(out, blobs, 9) == 0
        assert p.device_bytes()["digit_table"] == 0
