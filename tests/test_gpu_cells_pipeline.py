"""Cells of blobs (vkzg_b200_compute_cells_batch) from page-locked host buffers
at 16 blobs or more per chunk: the chunk runs as parts on side streams, each
copying in, computing and copying out.  Byte-exact against the pageable-buffer
path and, for a sample, the CPU oracle; a chunk holding an invalid blob returns
INVALID_BLOB and leaves that chunk's cells zeroed, since they went out before
the error words were read."""
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


def test_pinned_parts_match_pageable_and_oracle(oracle):
    torch = pytest.importorskip("torch")
    n = 80
    blobs = random_blobs(n, 818).reshape(n, BLOB)
    with vkzg_b200.Prover(max_batch_size=n) as p:
        want = np.frombuffer(p.compute_cells_batch(blobs.tobytes(), n), np.uint8)
        hb = _pinned(torch, blobs)
        hc = _pinned(torch, n_bytes=n * EXT, fill=0xAB)
        assert p.compute_cells_raw(hc.data_ptr(), hb.data_ptr(), n) == vkzg_b200.OK
        got = hc.numpy().copy()
    assert np.array_equal(got, want)
    pick = [0, 41, 79]
    rc, ref = oracle.compute_cells(np.ascontiguousarray(blobs[pick]))
    assert rc == 0
    assert np.array_equal(ref.reshape(-1), got.reshape(n, EXT)[pick].reshape(-1))


def test_pinned_parts_invalid_blob_zeroes_the_chunk(golden_proofs):
    torch = pytest.importorskip("torch")
    n = 72
    blobs = random_blobs(n, 819).reshape(n, BLOB)
    blobs[50] = golden_proofs["invalid_blob_0"].reshape(-1)
    with vkzg_b200.Prover(max_batch_size=n) as p:
        hb = _pinned(torch, blobs)
        hc = _pinned(torch, n_bytes=n * EXT, fill=0xAB)
        assert p.compute_cells_raw(hc.data_ptr(), hb.data_ptr(), n) == vkzg_b200.ERR_INVALID_BLOB
        assert not hc.numpy().any()
        # the prover stays usable: the valid blobs alone
        ok = np.delete(blobs, 50, axis=0)
        hb2 = _pinned(torch, ok)
        hc2 = _pinned(torch, n_bytes=(n - 1) * EXT)
        assert p.compute_cells_raw(hc2.data_ptr(), hb2.data_ptr(), n - 1) == vkzg_b200.OK
        want = np.frombuffer(p.compute_cells_batch(ok.tobytes(), n - 1), np.uint8)
        assert np.array_equal(hc2.numpy(), want)
