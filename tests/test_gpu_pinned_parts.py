"""Small and ragged chunks from page-locked host buffers.  From 16 blobs on, a
recovery or cells chunk runs as parts of at least 8 blobs on side streams
(copy in, kernel, copy out per part); 21 and 37 blobs give parts of unequal
length.  Recovery round-trips the blobs' cells; cells match the single-call
path from pageable memory and, for a sample, the CPU oracle.  Calls larger
than max_batch_size keep the chunk rule on these paths: chunks before a
failing one are written."""
import numpy as np
import pytest

import vkzg_b200
from conftest import random_blobs

pytestmark = pytest.mark.gpu

EXT = 128 * 2048
BLOB = 131072


def _pinned(torch, data=None, n_bytes=None, fill=0):
    t = torch.empty(n_bytes if data is None else data.size, dtype=torch.uint8).pin_memory()
    if data is None:
        t.fill_(fill)
    else:
        t.numpy()[:] = data.reshape(-1)
    return t


def _present(rng, n):
    pats = [np.r_[np.ones(64), np.zeros(64)], np.tile([0, 1], 64), np.ones(128)]
    while len(pats) < n:
        p = np.zeros(128)
        p[rng.choice(128, int(rng.integers(64, 128)), replace=False)] = 1
        pats.append(p)
    return np.stack(pats[:n]).astype(np.uint8)


@pytest.mark.parametrize("n", [16, 21, 37])
def test_pinned_cells_parts(n, oracle):
    torch = pytest.importorskip("torch")
    blobs = random_blobs(n, 900 + n).reshape(n, BLOB)
    with vkzg_b200.Prover(max_batch_size=64) as p:
        want = np.frombuffer(p.compute_cells_batch(blobs.tobytes(), n), np.uint8)
        hb = _pinned(torch, blobs)
        hc = _pinned(torch, n_bytes=n * EXT, fill=0xAB)
        assert p.compute_cells_raw(hc.data_ptr(), hb.data_ptr(), n) == vkzg_b200.OK
        got = hc.numpy().copy()
    assert np.array_equal(got, want)
    pick = [0, n - 1]
    rc, ref = oracle.compute_cells(np.ascontiguousarray(blobs[pick]))
    assert rc == 0
    assert np.array_equal(ref.reshape(-1), got.reshape(n, EXT)[pick].reshape(-1))


@pytest.mark.parametrize("n", [16, 21, 37])
def test_pinned_recovery_parts_round_trip(n, oracle):
    torch = pytest.importorskip("torch")
    blobs = random_blobs(n, 950 + n).reshape(n, BLOB)
    rng = np.random.default_rng(n)
    present = _present(rng, n)
    with vkzg_b200.Prover(max_batch_size=64) as p:
        cells = np.frombuffer(p.compute_cells_batch(blobs.tobytes(), n), np.uint8).reshape(n, 128, 2048)
        erased = cells.copy()
        erased[present == 0] = rng.integers(0, 256, size=erased[present == 0].shape, dtype=np.uint8)
        hi = _pinned(torch, erased)
        hp = _pinned(torch, present)
        ho = _pinned(torch, n_bytes=n * EXT, fill=0xCD)
        assert p.recover_cells_raw(ho.data_ptr(), hi.data_ptr(), hp.data_ptr(), n) == vkzg_b200.OK
        got = ho.numpy().reshape(n, 128, 2048).copy()
    assert np.array_equal(got, cells)
    rc, ref = oracle.compute_cells(np.ascontiguousarray(blobs[[n // 2]]))
    assert rc == 0
    assert np.array_equal(ref.reshape(-1), got[n // 2].reshape(-1))


def test_pinned_recovery_chunks_keep_earlier_on_error():
    """Chunks of max_batch_size blobs (16 here: 16, 16, 5), each run as parts: a
    blob with 65 cells missing in the second chunk returns BADARGS before that
    chunk's device work (src/vkzg.cpp:1093-1105), with the first chunk's cells
    written and the rest of the output untouched."""
    torch = pytest.importorskip("torch")
    n = 37
    blobs = random_blobs(n, 990).reshape(n, BLOB)
    rng = np.random.default_rng(99)
    present = _present(rng, n)
    present[20] = 0
    present[20, :63] = 1
    with vkzg_b200.Prover(max_batch_size=16) as p:
        cells = np.frombuffer(p.compute_cells_batch(blobs.tobytes(), n), np.uint8).reshape(n, 128, 2048)
        hi = _pinned(torch, cells)
        hp = _pinned(torch, present)
        ho = _pinned(torch, n_bytes=n * EXT, fill=0xCD)
        assert p.recover_cells_raw(ho.data_ptr(), hi.data_ptr(), hp.data_ptr(), n) == vkzg_b200.ERR_BADARGS
        got = ho.numpy().reshape(n, 128, 2048)
        assert np.array_equal(got[:16], cells[:16])
        assert (got[16:] == 0xCD).all()
        # the prover stays usable: the same call without the bad blob
        present[20, 63] = 1
        hp2 = _pinned(torch, present)
        assert p.recover_cells_raw(ho.data_ptr(), hi.data_ptr(), hp2.data_ptr(), n) == vkzg_b200.OK
        assert np.array_equal(ho.numpy().reshape(n, 128, 2048), cells)


def test_pinned_cells_chunks_keep_earlier_on_error(golden_proofs):
    """Cells in chunks of 16 (16, 16, 5) from page-locked buffers: an invalid blob
    in the second chunk leaves the first chunk's cells written, the second
    chunk's zeroed (its parts' cells went out before the error words were read)
    and the third untouched."""
    torch = pytest.importorskip("torch")
    n = 37
    blobs = random_blobs(n, 991).reshape(n, BLOB)
    blobs[21] = golden_proofs["invalid_blob_0"].reshape(-1)
    with vkzg_b200.Prover(max_batch_size=16) as p:
        want = np.frombuffer(p.compute_cells_batch(blobs[:16].tobytes(), 16), np.uint8)
        hb = _pinned(torch, blobs)
        hc = _pinned(torch, n_bytes=n * EXT, fill=0xAB)
        assert p.compute_cells_raw(hc.data_ptr(), hb.data_ptr(), n) == vkzg_b200.ERR_INVALID_BLOB
        got = hc.numpy()
        assert np.array_equal(got[:16 * EXT], want)
        assert not got[16 * EXT:32 * EXT].any()
        assert (got[32 * EXT:] == 0xAB).all()


@pytest.mark.parametrize("n", [16, 37])
@pytest.mark.parametrize("pin_in,pin_out", [(False, False), (True, False), (False, True)])
def test_pageable_recovery_parts_round_trip(n, pin_in, pin_out):
    """Pageable cells or output (16 blobs or more): 8-blob parts through the
    prover's pinned staging buffers, dealt to host threads; every combination of
    a pageable and a page-locked side recovers the blobs' cells."""
    torch = pytest.importorskip("torch")
    blobs = random_blobs(n, 970 + n).reshape(n, BLOB)
    rng = np.random.default_rng(n + 7)
    present = _present(rng, n)
    with vkzg_b200.Prover(max_batch_size=64) as p:
        cells = np.frombuffer(p.compute_cells_batch(blobs.tobytes(), n), np.uint8).reshape(n, 128, 2048)
        erased = cells.copy()
        erased[present == 0] = 0
        src = _pinned(torch, erased) if pin_in else np.ascontiguousarray(erased.reshape(-1))
        dst = _pinned(torch, n_bytes=n * EXT, fill=0xCD) if pin_out else np.full(n * EXT, 0xCD, np.uint8)
        src_ptr = src.data_ptr() if pin_in else src
        dst_ptr = dst.data_ptr() if pin_out else dst
        assert p.recover_cells_raw(dst_ptr, src_ptr, present, n) == vkzg_b200.OK
        got = (dst.numpy() if pin_out else dst).reshape(n, 128, 2048)
        assert np.array_equal(got, cells)


@pytest.mark.parametrize("n", [40, 100])
def test_pageable_proof_upload_parts(n, monkeypatch, oracle, mainnet_tables):
    """Pageable blobs (16 or more) go up through the pinned staging in parts
    dealt to host threads; 100 blobs take the two-piece path (parts of 9 blobs,
    the last of 1, each piece's front waiting for the parts that hold it), 40
    the single upload.  Proofs equal the page-locked call's and, for a sample,
    the CPU oracle's."""
    torch = pytest.importorskip("torch")
    monkeypatch.delenv("VKZG_TABLES_PATH", raising=False)
    monkeypatch.setenv("VKZG_PLAN", "3")
    monkeypatch.setenv("VKZG_COMB_WINDOWS", "26")
    blobs = random_blobs(n, 960 + n).reshape(n, BLOB)
    with vkzg_b200.Prover(max_batch_size=128) as p:
        out = np.zeros(n * 6144, np.uint8)
        for _ in range(2):  # the first call also captures the pipeline's graph
            out[:] = 0
            assert p.compute_proofs_raw(out, blobs, n) == vkzg_b200.OK
        hb = _pinned(torch, blobs)
        hp = _pinned(torch, n_bytes=n * 6144)
        assert p.compute_proofs_raw(hp.data_ptr(), hb.data_ptr(), n) == vkzg_b200.OK
        assert np.array_equal(out, hp.numpy())
    rc, want = oracle.compute_proofs(mainnet_tables, np.ascontiguousarray(blobs[[0, n - 1]]))
    assert rc == 0
    assert np.array_equal(want.reshape(-1), out.reshape(n, 6144)[[0, n - 1]].reshape(-1))


@pytest.mark.parametrize("n", [16, 37])
def test_pageable_cells_parts(n, golden_proofs):
    """Cells (and cells + proofs) with pageable blobs and output, 16 blobs or
    more: the blobs go up and the cells come down through the pinned staging in
    parts on host threads.  Bytes equal the page-locked call's; an invalid blob
    leaves a pageable output untouched (the cells come down only after the
    error words are read)."""
    torch = pytest.importorskip("torch")
    blobs = random_blobs(n, 940 + n).reshape(n, BLOB)
    with vkzg_b200.Prover(max_batch_size=64) as p:
        hb = _pinned(torch, blobs)
        hc = _pinned(torch, n_bytes=n * EXT)
        assert p.compute_cells_raw(hc.data_ptr(), hb.data_ptr(), n) == vkzg_b200.OK
        want = hc.numpy().copy()
        out = np.full(n * EXT, 0xAB, np.uint8)
        assert p.compute_cells_raw(out, np.ascontiguousarray(blobs.reshape(-1)), n) == vkzg_b200.OK
        assert np.array_equal(out, want)
        out[:] = 0xAB  # page-locked blobs, pageable cells
        assert p.compute_cells_raw(out, hb.data_ptr(), n) == vkzg_b200.OK
        assert np.array_equal(out, want)
        cells2 = np.zeros(n * EXT, np.uint8)
        proofs2 = np.zeros(n * 6144, np.uint8)
        assert p.compute_cells_and_proofs_raw(cells2, proofs2, np.ascontiguousarray(blobs.reshape(-1)), n) == vkzg_b200.OK
        assert np.array_equal(cells2, want)
        pw = np.zeros(n * 6144, np.uint8)
        assert p.compute_proofs_raw(pw, blobs, n) == vkzg_b200.OK
        assert np.array_equal(proofs2, pw)
        bad = blobs.copy()
        bad[n // 2] = golden_proofs["invalid_blob_0"].reshape(-1)
        out[:] = 0xAB
        assert p.compute_cells_raw(out, np.ascontiguousarray(bad.reshape(-1)), n) == vkzg_b200.ERR_INVALID_BLOB
        assert (out == 0xAB).all()
