"""The reference's end-to-end test (tests/test.cpp) through the C ABI on the GPU:
consensus-spec vectors, batching, API contract, chunking, concurrency, recovery."""
import ctypes
import os
import threading

import numpy as np
import pytest

import vkzg_b200
from conftest import recover_inputs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def prover():
    os.environ.pop("VKZG_TABLES_PATH", None)
    p = vkzg_b200.Prover(max_batch_size=4)  # tests/test.cpp:35
    yield p
    p.close()


def test_device(prover):
    assert prover.device_name()
    assert prover.gpu_core_count() > 0
    assert prover.tables_source().startswith(("generated:", "file:"))


def test_proof_vectors(prover, golden_proofs):
    """tests/test.cpp:55-91"""
    for k, name in enumerate(golden_proofs["valid_names"]):
        out = prover.compute_cell_kzg_proofs_batch(golden_proofs["valid_blobs"][k].tobytes(), 1)
        assert out == golden_proofs["valid_proofs"][k].tobytes(), name


def test_invalid_blobs(prover, golden_proofs):
    for k, name in enumerate(golden_proofs["invalid_names"]):
        blob = golden_proofs[f"invalid_blob_{k}"]
        if blob.size != 131072:
            continue
        with pytest.raises(vkzg_b200.VkzgException) as e:
            prover.compute_cell_kzg_proofs_batch(blob.tobytes(), 1)
        assert e.value.code == vkzg_b200.ERR_INVALID_BLOB, name


def test_proof_vectors_batched(prover, golden_proofs):
    """tests/test.cpp:94-119 (7 blobs: two chunks of max_batch_size 4)"""
    blobs = golden_proofs["valid_blobs"]
    out = prover.compute_cell_kzg_proofs_batch(blobs.tobytes(), len(blobs))
    assert out == golden_proofs["valid_proofs"].tobytes()


def test_api_contract(prover, golden_proofs):
    """tests/test.cpp:122-171"""
    L = vkzg_b200.library()
    blob = np.ascontiguousarray(golden_proofs["valid_blobs"][3])
    want = golden_proofs["valid_proofs"][3].tobytes()
    proofs = np.zeros(6144, np.uint8)
    h = prover.handle
    assert L.vkzg_compute_proofs_batch(None, proofs.ctypes.data, blob.ctypes.data, 1) == 1
    assert L.vkzg_compute_proofs_batch(h, proofs.ctypes.data, None, 1) == 1
    assert L.vkzg_compute_proofs_batch(h, None, blob.ctypes.data, 1) == 1
    assert L.vkzg_compute_proofs_batch(h, proofs.ctypes.data, blob.ctypes.data, 0) == 0
    big = 4 * 2 + 1
    blobs = np.tile(blob, big)
    out = np.zeros(big * 6144, np.uint8)
    assert prover.compute_proofs_raw(out, blobs, big) == 0
    for i in range(big):
        assert out[i * 6144:(i + 1) * 6144].tobytes() == want


def test_invalid_blob_in_later_chunk_keeps_earlier_chunks(prover, golden_proofs):
    """Chunk-level error semantics (src/vkzg.cpp:1191-1197): chunks before the bad one are written."""
    good = golden_proofs["valid_blobs"][2]
    bad = golden_proofs["invalid_blob_1"]
    blobs = np.concatenate([np.tile(good, 4), bad, good])
    out = np.zeros(6 * 6144, np.uint8)
    assert prover.compute_proofs_raw(out, blobs, 6) == vkzg_b200.ERR_INVALID_BLOB
    for i in range(4):
        assert out[i * 6144:(i + 1) * 6144].tobytes() == golden_proofs["valid_proofs"][2].tobytes()
    assert not out[4 * 6144:].any()


def test_concurrent_calls(prover, golden_proofs):
    """tests/test.cpp:175-202: 4 threads x 3 calls on one prover."""
    bad = []

    def work(t):
        for r in range(3):
            k = (t + r) % len(golden_proofs["valid_names"])
            out = prover.compute_cell_kzg_proofs_batch(golden_proofs["valid_blobs"][k].tobytes(), 1)
            if out != golden_proofs["valid_proofs"][k].tobytes():
                bad.append((t, r))

    threads = [threading.Thread(target=work, args=(t,)) for t in range(4)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not bad


def test_recovery_vectors(prover, golden_recover):
    """tests/test.cpp:205-276: each vector alone, then all valid ones batched."""
    valid = []
    for name in golden_recover["names"]:
        full, present = recover_inputs(golden_recover, name)
        if name + "__expected" in golden_recover.files:
            out = prover.recover_cells_batch(full.tobytes(), present.tobytes(), 1)
            assert out == golden_recover[name + "__expected"].tobytes(), name
            valid.append((full, present, golden_recover[name + "__expected"]))
        else:
            with pytest.raises(vkzg_b200.VkzgException) as e:
                prover.recover_cells_batch(full.tobytes(), present.tobytes(), 1)
            assert e.value.code == vkzg_b200.ERR_BADARGS, name
    cells = np.concatenate([v[0] for v in valid])
    present = np.concatenate([v[1] for v in valid])
    out = prover.recover_cells_batch(cells.tobytes(), present.tobytes(), len(valid))
    assert out == np.concatenate([v[2] for v in valid]).tobytes()


def test_stage_timing(prover, golden_proofs):
    prover.set_stage_timing(True)
    prover.compute_cell_kzg_proofs_batch(golden_proofs["valid_blobs"][2].tobytes(), 1)
    t = prover.last_stage_times()
    prover.set_stage_timing(False)
    assert len(t) == 10 and all(v >= 0 for v in t.values()) and sum(t.values()) > 0


def test_java_style_global_api(golden_proofs):
    """The module-level mirror of Vkzg.java (init / computeCellKzgProofsBatch / deinit)."""
    vkzg_b200.init(2)
    try:
        with pytest.raises(RuntimeError):
            vkzg_b200.init()
        assert vkzg_b200.gpuCoreCount() > 0
        out = vkzg_b200.computeCellKzgProofsBatch(golden_proofs["valid_blobs"][5].tobytes(), 1)
        assert out == golden_proofs["valid_proofs"][5].tobytes()
        with pytest.raises(ValueError):
            vkzg_b200.computeCellKzgProofsBatch(b"\0" * 10, 1)
    finally:
        vkzg_b200.deinit()


def test_cells_vectors(prover, golden_proofs):
    """The vectors' 128 cells (present in tests/vectors, skipped by tests/vectors.h:88-95)."""
    import hashlib
    blobs = golden_proofs["valid_blobs"]
    cells = prover.compute_cells_batch(blobs.tobytes(), len(blobs))
    for k in range(len(blobs)):
        digest = hashlib.sha256(cells[k * 262144:(k + 1) * 262144]).digest()
        assert digest == golden_proofs["valid_cells_sha256"][k].tobytes(), k
    cells2, proofs = prover.compute_cells_and_kzg_proofs_batch(blobs.tobytes(), len(blobs))
    assert cells2 == cells
    assert proofs == golden_proofs["valid_proofs"].tobytes()
    with pytest.raises(vkzg_b200.VkzgException) as e:
        prover.compute_cells_batch(golden_proofs["invalid_blob_0"].tobytes(), 1)
    assert e.value.code == vkzg_b200.ERR_INVALID_BLOB


def test_cells_then_recover_roundtrip(prover, golden_proofs):
    """compute_cells -> erase half -> recover gives the cells back (size-independent check)."""
    blobs = golden_proofs["valid_blobs"][2:5]
    cells = np.frombuffer(prover.compute_cells_batch(blobs.tobytes(), 3), np.uint8).reshape(3, 128, 2048).copy()
    present = np.ones((3, 128), np.uint8)
    present[0, 64:] = 0
    present[1, ::2] = 0
    present[2, [3, 9, 77]] = 0
    erased = cells.copy()
    erased[present == 0] = 0x5A
    out = prover.recover_cells_batch(erased.tobytes(), present.tobytes(), 3)
    assert out == cells.tobytes()


def test_recovery_vectors_with_proofs(prover, golden_recover):
    """recover_cells_and_kzg_proofs: cells and the recovered blob's proofs (output[1] of the
    recovery vectors, which tests/vectors.h:8-10 leaves unchecked)."""
    names = [n for n in golden_recover["names"] if n + "__expected" in golden_recover.files]
    ins = [recover_inputs(golden_recover, n) for n in names]
    cells = np.concatenate([c for c, _ in ins])
    present = np.concatenate([p for _, p in ins])
    out, proofs = prover.recover_cells_and_kzg_proofs_batch(cells.tobytes(), present.tobytes(), len(names))
    for k, n in enumerate(names):
        assert out[k * 262144:(k + 1) * 262144] == golden_recover[n + "__expected"].tobytes(), n
        assert proofs[k * 6144:(k + 1) * 6144] == golden_recover[n + "__proofs"].tobytes(), n
