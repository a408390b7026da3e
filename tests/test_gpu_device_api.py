"""The device-pointer entry points (vkzg_b200_compute_proofs_device /
vkzg_b200_recover_cells_device) on torch CUDA buffers and a caller stream:
same bytes as the host entry points, chunked beyond max_batch_size, per-blob
error words, ordering on the caller's stream."""
import numpy as np
import pytest

import vkzg_b200
from conftest import adversarial_blobs, random_blobs

pytestmark = pytest.mark.gpu


def test_device_proofs_match_host_and_flag_bad_blobs():
    import torch
    dev = torch.device("cuda", 0)
    blobs = np.concatenate([random_blobs(36, 909), adversarial_blobs()])  # 40 blobs
    bad = blobs.copy()
    bad[7, :32] = 0xFF  # non-canonical element in blob 7
    n = len(blobs)
    with vkzg_b200.Prover(max_batch_size=32) as p:  # two chunks
        want = np.zeros(n * 6144, np.uint8)
        assert p.compute_proofs_raw(want, blobs, n) == 0
        stream = torch.cuda.Stream(dev)
        with torch.cuda.stream(stream):
            d_blobs = torch.from_numpy(bad).to(dev, non_blocking=False)
            d_out = torch.zeros(n * 6144, dtype=torch.uint8, device=dev)
            d_err = torch.full((n,), 7, dtype=torch.int32, device=dev)
        assert p.compute_proofs_device(d_out.data_ptr(), d_blobs.data_ptr(), d_err.data_ptr(), n,
                                       stream.cuda_stream) == 0
        with torch.cuda.stream(stream):
            got = d_out.cpu().numpy()  # ordered after the proofs on the caller's stream
            err = d_err.cpu().numpy()
    assert err[7] != 0 and int(np.count_nonzero(err)) == 1
    for b in range(n):
        if b != 7:
            assert np.array_equal(got[b * 6144:(b + 1) * 6144], want[b * 6144:(b + 1) * 6144]), b


def test_device_recovery_matches_host():
    import torch
    dev = torch.device("cuda", 0)
    n = 20
    rng = np.random.default_rng(4)
    blobs = random_blobs(n, 808)
    with vkzg_b200.Prover(max_batch_size=16) as p:
        cells = np.frombuffer(p.compute_cells_batch(blobs.tobytes(), n), np.uint8).reshape(n, 128, 2048)
        present = np.ones((n, 128), np.uint8)
        for b in range(n):
            present[b, rng.choice(128, int(rng.integers(0, 65)), replace=False)] = 0
        present[3, :65] = 0  # too many missing: its error word, the others unaffected
        erased = cells.copy()
        erased[present == 0] = 0
        d_cells = torch.from_numpy(erased.reshape(-1)).to(dev)
        d_present = torch.from_numpy(present.reshape(-1)).to(dev)
        d_out = torch.zeros(n * 262144, dtype=torch.uint8, device=dev)
        d_err = torch.zeros(n, dtype=torch.int32, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        assert p.recover_cells_device(d_out.data_ptr(), d_cells.data_ptr(), d_present.data_ptr(),
                                      d_err.data_ptr(), n, stream) == 0
        got = d_out.cpu().numpy().reshape(n, -1)
        err = d_err.cpu().numpy()
    assert err[3] != 0 and int(np.count_nonzero(err)) == 1
    for b in range(n):
        if b != 3:
            assert np.array_equal(got[b], cells[b].reshape(-1)), b
