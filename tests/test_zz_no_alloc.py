"""Allocation-free recovery entry point (vkzg_b200_recover_cells_device_noalloc).

Some callers cannot allocate device memory when they call in: a framework's
memory pool may already own nearly all of HBM, a latency-critical loop cannot
absorb the synchronisation a cudaMalloc/cudaFree implies, and code enqueueing on
a stream it does not own must not add allocations to it.  This entry point runs
recovery with no scratch: each blob's cluster of four blocks keeps its working
state in shared memory.

The test calls it through the C ABI twice in a row, on different inputs, and
checks each output byte for byte against the CPU oracle's recovery of the same
inputs (an independent restatement: per-element Fermat division, separate
transforms), and against the existing device entry point.  Recovery is exact
integer work, so the tolerance is zero.  A blob with more than 64 cells missing
must get a nonzero error word while the others in the same call still recover.
The test builds its own prover and inputs, so it passes alone in a fresh process
as well as after the other tests.
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


def _device_call(torch, prover, fn, cells_np, present_np, fill):
    dev = torch.device("cuda", 0)
    n = len(present_np)
    cells = torch.from_numpy(np.ascontiguousarray(cells_np)).to(dev)
    present = torch.from_numpy(np.ascontiguousarray(present_np)).to(dev)
    out = torch.full((n * EXT,), fill, dtype=torch.uint8, device=dev)
    err = torch.full((n,), 7, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = fn(out.data_ptr(), cells.data_ptr(), present.data_ptr(), err.data_ptr(), n, stream)
    torch.cuda.synchronize()
    return rc, out.cpu().numpy(), err.cpu().numpy()


def test_noalloc_recovery_matches_oracle(oracle):
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    prover = vkzg_b200.Prover(max_batch_size=vkzg_b200.NOALLOC_MAX_BLOBS)
    try:
        for call, (n, seed) in enumerate([(5, 11), (vkzg_b200.NOALLOC_MAX_BLOBS, 12)]):
            cells, present = _inputs(n, seed)
            orc, want = oracle.recover_cells(cells, present)
            assert orc == 0
            rc, got, err = _device_call(torch, prover, prover.recover_cells_device_noalloc, cells, present, 0xEE)
            assert rc == 0, f"call {call}: status {rc}"
            assert not err.any(), f"call {call}: error words {err}"
            assert np.array_equal(got, want), f"call {call}: output differs from the oracle"
            rc, via_device, _ = _device_call(torch, prover, prover.recover_cells_device, cells, present, 0)
            assert rc == 0 and np.array_equal(via_device, got)
    finally:
        prover.close()


def test_noalloc_flags_blob_with_too_few_cells(oracle):
    torch = pytest.importorskip("torch")
    torch.cuda.set_device(0)
    prover = vkzg_b200.Prover(max_batch_size=4)
    try:
        cells, present = _inputs(3, 13)
        present[1] = 0
        present[1, 3::2] = 1  # 63 present, 65 missing
        rc, got, err = _device_call(torch, prover, prover.recover_cells_device_noalloc, cells, present, 0)
        assert rc == 0
        assert err[1] != 0 and err[0] == 0 and err[2] == 0
        for b in (0, 2):
            orc, want = oracle.recover_cells(cells[b], present[b])
            assert orc == 0 and np.array_equal(got[b * EXT:(b + 1) * EXT], want)
    finally:
        prover.close()


def test_noalloc_rejects_more_blobs_than_its_limit():
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
