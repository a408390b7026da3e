"""GPU path against the CPU oracle on seeded synthetic inputs: tables generated
on the device, proofs for random and adversarial blobs under a synthetic setup,
recovery with uneven survivor sets, non-canonical and garbage cells."""
import os

import numpy as np
import pytest

import vkzg_b200
from conftest import adversarial_blobs, random_blobs

pytestmark = pytest.mark.gpu


def test_device_tables_match_oracle(oracle, mainnet_tables, mainnet_setup, tmp_path):
    """Tables generated on the GPU are byte-identical to the oracle's."""
    path = str(tmp_path / "tables.bin")
    vkzg_b200.write_tables(mainnet_setup, path)
    got = np.fromfile(path, np.uint8)
    want = mainnet_tables.serialize()
    assert got.size == want.size
    assert np.array_equal(got, want)


def test_tables_cache_file(mainnet_tables, golden_proofs, tmp_path, monkeypatch):
    """$VKZG_TABLES_CACHE: the first prover generates the tables and writes them
    there (the oracle's bytes); the next one loads that file and proves the same."""
    cache = str(tmp_path / "cache.bin")
    monkeypatch.delenv("VKZG_TABLES_PATH", raising=False)
    monkeypatch.setenv("VKZG_TABLES_CACHE", cache)
    blob = golden_proofs["valid_blobs"][1].tobytes()
    with vkzg_b200.Prover(max_batch_size=1) as p1:
        assert p1.tables_source().startswith("generated:") and cache in p1.tables_source()
        first = p1.compute_cell_kzg_proofs_batch(blob, 1)
    assert np.array_equal(np.fromfile(cache, np.uint8), mainnet_tables.serialize())
    with vkzg_b200.Prover(max_batch_size=1) as p2:
        assert p2.tables_source() == "file:" + cache
        assert p2.compute_cell_kzg_proofs_batch(blob, 1) == first == golden_proofs["valid_proofs"][1].tobytes()


@pytest.fixture(scope="module")
def synthetic_prover(synthetic, tmp_path_factory):
    tau, mono, tables = synthetic
    path = str(tmp_path_factory.mktemp("synth") / "tables.bin")
    vkzg_b200.write_tables(mono, path)
    os.environ["VKZG_TABLES_PATH"] = path
    try:
        p = vkzg_b200.Prover(max_batch_size=16)
    finally:
        os.environ.pop("VKZG_TABLES_PATH", None)
    assert p.tables_source() == "file:" + path
    yield p
    p.close()


def test_synthetic_proofs_vs_oracle(synthetic, synthetic_prover, oracle):
    tau, mono, tables = synthetic
    blobs = np.concatenate([random_blobs(6, 101), adversarial_blobs()])
    out = np.zeros(len(blobs) * 6144, np.uint8)
    assert synthetic_prover.compute_proofs_raw(out, blobs, len(blobs)) == 0
    rc, want = oracle.compute_proofs(tables, blobs)
    assert rc == 0
    for b in range(len(blobs)):
        assert np.array_equal(out[b * 6144:(b + 1) * 6144], want[b * 6144:(b + 1) * 6144]), b
    rc, direct = oracle.compute_proofs_tau(tau, blobs[0])
    assert np.array_equal(out[:6144], direct)


def _patterns(rng, n):
    pats = [np.r_[np.ones(64), np.zeros(64)], np.r_[np.zeros(64), np.ones(64)],
            np.tile([1, 0], 64), np.ones(128)]
    while len(pats) < n:
        keep = int(rng.integers(64, 128))
        p = np.zeros(128)
        p[rng.choice(128, keep, replace=False)] = 1
        pats.append(p)
    return np.stack(pats[:n]).astype(np.uint8)


def test_recovery_vs_oracle(synthetic_prover, oracle):
    n = 12
    blobs = random_blobs(n, 202)
    rc, cells = oracle.compute_cells(blobs)
    assert rc == 0
    rng = np.random.default_rng(77)
    present = _patterns(rng, n)
    inp = cells.reshape(n, 128, 2048).copy()
    inp[present == 0] = rng.integers(0, 256, size=inp[present == 0].shape, dtype=np.uint8)  # ignored
    out = np.zeros(n * 262144, np.uint8)
    assert synthetic_prover.recover_cells_raw(out, inp, present, n) == 0
    assert np.array_equal(out, cells)


def test_recovery_inconsistent_and_noncanonical_vs_oracle(synthetic_prover, oracle):
    """Inputs that are not a codeword, with present cells >= r: the GPU computes
    the same linear map as the reference (values mod r)."""
    rng = np.random.default_rng(5)
    n = 3
    cells = rng.integers(0, 256, size=(n, 128, 2048), dtype=np.uint8)
    present = _patterns(rng, 4 + n)[4:]
    out = np.zeros(n * 262144, np.uint8)
    assert synthetic_prover.recover_cells_raw(out, cells, present, n) == 0
    rc, want = oracle.recover_cells(cells, present)
    assert rc == 0
    assert np.array_equal(out, want)


def test_recovery_too_many_missing(synthetic_prover):
    cells = np.zeros((2, 128, 2048), np.uint8)
    present = np.ones((2, 128), np.uint8)
    present[1, :65] = 0
    out = np.zeros(2 * 262144, np.uint8)
    assert synthetic_prover.recover_cells_raw(out, cells, present, 2) == vkzg_b200.ERR_BADARGS


def test_graph_replay_matches_direct_launches(monkeypatch):
    """Chunks replayed from the captured CUDA graph give the same bytes as the
    same pipeline launched kernel by kernel, and count the same launches."""
    monkeypatch.delenv("VKZG_TABLES_PATH", raising=False)
    blobs = np.concatenate([random_blobs(10, 505), adversarial_blobs()])
    outs, counts = [], []
    for graphs in ("0", "1"):
        monkeypatch.setenv("VKZG_GRAPHS", graphs)
        with vkzg_b200.Prover(max_batch_size=len(blobs)) as p:
            out = np.zeros(len(blobs) * 6144, np.uint8)
            assert p.compute_proofs_raw(out, blobs, len(blobs)) == 0  # first call: tuning, capture
            for _ in range(2):
                before = vkzg_b200.kernel_launches()
                out2 = np.zeros_like(out)
                assert p.compute_proofs_raw(out2, blobs, len(blobs)) == 0
                counts.append(vkzg_b200.kernel_launches() - before)
                assert np.array_equal(out, out2)
            outs.append(out)
    assert np.array_equal(outs[0], outs[1])
    assert counts[0] == counts[1] == counts[2] == counts[3] > 0
