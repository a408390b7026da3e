"""Faults injected on the host: missing, truncated and corrupted setup files
(the status codes of src/precomputed_tables.cpp:16-73 and src/vkzg.cpp:170-181),
and the serving loop under a one-byte HBM admission budget and a zero wait
timeout.  Nothing here faults the device: every failure is a file or a
host-side limit."""
import numpy as np
import pytest

import vkzg_b200

pytestmark = pytest.mark.gpu

_TAIL_PERM_BYTES = 2 * 128 * 4 + 32  # perm[2][128] u32, then the 32-byte 1/4096


def _prover_status(monkeypatch, tables, setup):
    """Status of vkzg_prover_new with only the given table file and setup file."""
    monkeypatch.delenv("VKZG_TABLES_CACHE", raising=False)
    monkeypatch.setenv("VKZG_TABLES_PATH", tables)
    monkeypatch.setenv("VKZG_SETUP_PATH", setup)
    try:
        p = vkzg_b200.Prover(max_batch_size=1)
    except vkzg_b200.VkzgException as e:
        return e.code, None
    return vkzg_b200.OK, p


@pytest.fixture
def table_bytes(mainnet_tables):
    return bytearray(mainnet_tables.serialize())


def test_no_tables_and_no_setup_is_io(tmp_path, monkeypatch):
    rc, _ = _prover_status(monkeypatch, str(tmp_path / "absent.bin"), str(tmp_path / "absent_setup.bin"))
    assert rc == vkzg_b200.ERR_IO


@pytest.mark.parametrize("fault", ["truncated", "magic", "version", "perm", "offsets", "item_digit"])
def test_malformed_tables_file_is_setup(fault, table_bytes, tmp_path, monkeypatch):
    b = table_bytes
    words = np.frombuffer(b, np.uint32, count=4)
    n0, n1 = int(words[2]), int(words[3])
    perm0 = len(b) - _TAIL_PERM_BYTES
    offsets0 = perm0 - 2 * 129 * 4
    items0 = offsets0 - 4 * (n0 + n1)
    if fault == "truncated":
        b = b[: len(b) // 2]
    elif fault == "magic":
        b[0] ^= 0xFF
    elif fault == "version":
        b[4:8] = (2).to_bytes(4, "little")
    elif fault == "perm":
        b[perm0:perm0 + 4] = (200).to_bytes(4, "little")  # a bucket index >= 128
    elif fault == "offsets":
        b[offsets0 + 4:offsets0 + 8] = (n0 + 1).to_bytes(4, "little")  # not monotone up to n0
    elif fault == "item_digit":
        word = int.from_bytes(b[items0:items0 + 4], "little")
        b[items0:items0 + 4] = ((word & ~0xFF00) | (40 << 8)).to_bytes(4, "little")  # digit row 40 >= 32
    path = tmp_path / "tables.bin"
    path.write_bytes(bytes(b))
    rc, _ = _prover_status(monkeypatch, str(path), str(tmp_path / "absent_setup.bin"))
    assert rc == vkzg_b200.ERR_SETUP, fault


def test_short_setup_file_is_setup(mainnet_setup, tmp_path, monkeypatch):
    setup = tmp_path / "setup.bin"
    setup.write_bytes(mainnet_setup[:-48])
    rc, _ = _prover_status(monkeypatch, str(tmp_path / "absent.bin"), str(setup))
    assert rc == vkzg_b200.ERR_SETUP


def test_truncated_tables_fall_back_to_generation(table_bytes, mainnet_setup, golden_proofs, tmp_path, monkeypatch):
    """A malformed table file with a readable setup behind it: the prover generates
    the tables on the device and proves the golden vector."""
    path = tmp_path / "tables.bin"
    path.write_bytes(bytes(table_bytes[:1000]))
    setup = tmp_path / "setup.bin"
    setup.write_bytes(mainnet_setup)
    rc, p = _prover_status(monkeypatch, str(path), str(setup))
    assert rc == vkzg_b200.OK
    with p:
        assert p.tables_source() == "generated:" + str(setup)
        blob = golden_proofs["valid_blobs"][2].tobytes()
        assert p.compute_cell_kzg_proofs_batch(blob, 1) == golden_proofs["valid_proofs"][2].tobytes()


def test_server_one_byte_budget_still_serves_every_request(golden_proofs, golden_recover):
    """An admission budget below one batch admits one batch at a time (a batch is
    always admitted when nothing is in flight) and every request completes."""
    from conftest import recover_inputs

    blobs = golden_proofs["valid_blobs"]
    want_p = golden_proofs["valid_proofs"].reshape(-1)
    name = [n for n in golden_recover["names"] if n + "__expected" in golden_recover.files][1]
    cells, present = recover_inputs(golden_recover, name)
    want_r = golden_recover[name + "__expected"]
    with vkzg_b200.Server(max_blobs_per_batch=4, lanes=2, hbm_budget_bytes=1) as s:
        jobs = []
        for k in range(6):
            if k % 3 == 2:
                out = np.zeros(want_r.size, np.uint8)
                jobs.append((s.submit_recovery(out, cells, present, 1), out, want_r))
            else:
                out = np.zeros(want_p.size, np.uint8)
                jobs.append((s.submit_proofs(out, blobs, len(blobs)), out, want_p))
        for t, out, want in jobs:
            assert s.wait(t) == vkzg_b200.OK
            assert np.array_equal(out, want)
        st = s.stats()
        assert st["requests"] == len(jobs)
        assert st["proof_bytes_per_blob"] > st["recover_bytes_per_blob"] > 0
        assert st["resident_bytes"] > 0


def test_server_budget_binding_partway(golden_proofs):
    """A budget of one and a half full proof batches: a second batch is admitted
    only while the first is small enough; the dispatcher defers the rest, the
    in-flight charge never exceeds the budget once something is in flight, and
    every request completes with the right bytes."""
    from conftest import random_blobs
    blobs = random_blobs(16, 717)
    with vkzg_b200.Prover(max_batch_size=16) as p:
        want = np.frombuffer(p.compute_cell_kzg_proofs_batch(blobs.tobytes(), 16), np.uint8)
    with vkzg_b200.Server(max_blobs_per_batch=8, lanes=3) as probe:
        per_blob = probe.stats()["proof_bytes_per_blob"]
    budget = int(per_blob * 8 * 1.5)
    with vkzg_b200.Server(max_blobs_per_batch=8, lanes=3, hbm_budget_bytes=budget) as s:
        jobs = []
        for k in range(24):
            out = np.zeros(16 * 6144, np.uint8)
            jobs.append((s.submit_proofs(out, blobs, 16), out))
        for t, out in jobs:
            assert s.wait(t) == vkzg_b200.OK
            assert np.array_equal(out, want)
        st = s.stats()
        assert st["requests"] == 24
        assert st["deferrals"] > 0
        assert st["peak_in_flight_bytes"] <= budget


def test_server_wait_timeout_keeps_ticket(golden_proofs):
    """wait() with a zero timeout on a request still in flight returns PENDING and
    the ticket stays valid; a spent or unknown ticket is BADARGS."""
    blobs = np.tile(golden_proofs["valid_blobs"], (10, 1))
    with vkzg_b200.Server(max_blobs_per_batch=64) as s:
        out = np.zeros(len(blobs) * 6144, np.uint8)
        t = s.submit_proofs(out, blobs, len(blobs))
        rc = s.wait(t, 0)
        assert rc in (vkzg_b200.PENDING, vkzg_b200.OK)
        if rc == vkzg_b200.PENDING:
            assert t in s._keep
            assert s.wait(t) == vkzg_b200.OK
        assert t not in s._keep
        assert s.wait(t) == vkzg_b200.ERR_BADARGS
        assert s.wait(t + 1000) == vkzg_b200.ERR_BADARGS
        want = np.tile(golden_proofs["valid_proofs"], (10, 1)).reshape(-1)
        assert np.array_equal(out, want)
