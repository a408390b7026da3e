"""Allocation-free recovery entry point (vkzg_b200_recover_cells_device_noalloc).

Some callers cannot allocate device memory when they call in: a framework's
memory pool may already own nearly all of HBM, a latency-critical loop cannot
absorb the synchronisation a cudaMalloc/cudaFree implies, and code enqueueing on
a stream it does not own must not add allocations to it.  This entry point runs
recovery with no scratch: each blob's cluster of four blocks keeps its working
state in shared memory.

The test calls it through the C ABI twice in a row, on different inputs, and
checks each output byte for byte against the existing device entry point
(vkzg_b200_recover_cells_device, which uses the prover's cudaMalloc'd working
set).  Recovery is exact integer work, so the tolerance is zero.  It builds its
own prover and inputs, so it passes alone in a fresh process as well as after
the other tests.
"""
import numpy as np
import pytest

import vkzg_b200

pytestmark = pytest.mark.gpu

EXT = 128 * 2048


def _inputs(n, seed):
    """Random canonical cells (not a codeword: the recovery map is exercised on
    arbitrary values) and presence masks with 64..128 survivors, including the
    first-half and every-other patterns."""
    rng = np.random.default_rng(seed)
    cells = rng.integers(0, 256, size=(n, 8192, 32), dtype=np.uint8)
    cells[:, :, 0] &= 0x3F
    present = np.zeros((n, 128), np.uint8)
    for b in range(n):
        if b == 0:
            present[b, :64] = 1
        elif b == 1:
            present[b, ::2] = 1
        else:
            present[b, rng.choice(128, int(rng.integers(64, 129)), replace=False)] = 1
    return cells.reshape(n, EXT), present


def test_noalloc_recovery_matches_device_entry_point():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    prover = vkzg_b200.Prover(max_batch_size=vkzg_b200.NOALLOC_MAX_BLOBS)
    stream = torch.cuda.current_stream(dev).cuda_stream
    try:
        for call, (n, seed) in enumerate([(5, 11), (vkzg_b200.NOALLOC_MAX_BLOBS, 12)]):
            cells_np, present_np = _inputs(n, seed)
            cells = torch.from_numpy(cells_np).to(dev)
            present = torch.from_numpy(present_np).to(dev)
            out_ref = torch.zeros(n * EXT, dtype=torch.uint8, device=dev)
            out_new = torch.full((n * EXT,), 0xEE, dtype=torch.uint8, device=dev)
            err_ref = torch.full((n,), 7, dtype=torch.int32, device=dev)
            err_new = torch.full((n,), 7, dtype=torch.int32, device=dev)
            rc = prover.recover_cells_device(out_ref.data_ptr(), cells.data_ptr(), present.data_ptr(),
                                             err_ref.data_ptr(), n, stream)
            assert rc == 0
            rc = prover.recover_cells_device_noalloc(out_new.data_ptr(), cells.data_ptr(), present.data_ptr(),
                                                     err_new.data_ptr(), n, stream)
            assert rc == 0, f"call {call}: status {rc}"
            torch.cuda.synchronize()
            assert int(err_new.count_nonzero()) == 0 and int(err_ref.count_nonzero()) == 0
            assert torch.equal(out_new, out_ref), f"call {call}: outputs differ"
    finally:
        prover.close()


def test_noalloc_rejects_more_than_its_scratch_holds():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    prover = vkzg_b200.Prover(max_batch_size=2)
    try:
        n = vkzg_b200.NOALLOC_MAX_BLOBS + 1
        cells = torch.zeros(n * EXT, dtype=torch.uint8, device=dev)
        present = torch.ones(n * 128, dtype=torch.uint8, device=dev)
        out = torch.zeros(n * EXT, dtype=torch.uint8, device=dev)
        err = torch.zeros(n, dtype=torch.int32, device=dev)
        rc = prover.recover_cells_device_noalloc(out.data_ptr(), cells.data_ptr(), present.data_ptr(),
                                                 err.data_ptr(), n, None)
        assert rc == vkzg_b200.ERR_BADARGS
    finally:
        prover.close()
