"""Serving loop (vkzg_b200_server_*): continuous batching across lanes.  Every
request's output must be the same alone and in the mix, requests larger than
a batch are split, and a bad request fails alone."""
import numpy as np
import pytest

import vkzg_b200

pytestmark = pytest.mark.gpu


def test_mix_equals_alone(golden_proofs, golden_recover):
    from conftest import random_blobs, recover_inputs
    rng = np.random.default_rng(31)
    blobs = random_blobs(24, 77)
    # reference outputs: each request alone through the blocking C ABI
    with vkzg_b200.Prover(max_batch_size=32) as p:
        alone_proofs = np.frombuffer(p.compute_cell_kzg_proofs_batch(blobs.tobytes(), 24), np.uint8).reshape(24, 6144)
        cells = np.frombuffer(p.compute_cells_batch(blobs.tobytes(), 24), np.uint8).reshape(24, 262144)
    present = np.ones((24, 128), np.uint8)
    for b in range(24):
        present[b, rng.choice(128, int(rng.integers(0, 65)), replace=False)] = 0
    erased = cells.reshape(24, 128, 2048).copy()
    erased[present == 0] = 0x33
    erased = erased.reshape(24, 262144)

    # requests of uneven sizes, proofs and recoveries interleaved, one larger than a batch
    sizes = [1, 5, 9, 2, 7]
    reqs, start = [], 0
    for n in sizes:
        reqs.append(("proofs", start, n))
        reqs.append(("recover", start, n))
        start = (start + n) % 20
    bad = blobs[:2].copy()
    bad[1, :32] = 0xFF  # non-canonical element
    with vkzg_b200.Server(max_blobs_per_batch=8, lanes=2) as srv:
        outs, tickets = [], []
        for kind, s0, n in reqs:
            if kind == "proofs":
                out = np.zeros(n * 6144, np.uint8)
                t = srv.submit_proofs(out, np.ascontiguousarray(blobs[s0:s0 + n]), n)
            else:
                out = np.zeros(n * 262144, np.uint8)
                t = srv.submit_recovery(out, np.ascontiguousarray(erased[s0:s0 + n]),
                                        np.ascontiguousarray(present[s0:s0 + n]), n)
            outs.append(out)
            tickets.append(t)
        bad_out = np.zeros(2 * 6144, np.uint8)
        bad_t = srv.submit_proofs(bad_out, bad, 2)
        big = np.zeros(20 * 6144, np.uint8)  # 20 blobs > max_blobs_per_batch: split into parts
        big_t = srv.submit_proofs(big, np.ascontiguousarray(blobs[:20]), 20)
        for (kind, s0, n), out, t in zip(reqs, outs, tickets):
            assert srv.wait(t) == 0
            if kind == "proofs":
                assert np.array_equal(out.reshape(n, 6144), alone_proofs[s0:s0 + n]), (kind, s0, n)
            else:
                assert np.array_equal(out.reshape(n, 262144), cells[s0:s0 + n]), (kind, s0, n)
        assert srv.wait(bad_t) == vkzg_b200.ERR_INVALID_BLOB
        assert srv.wait(big_t) == 0
        assert np.array_equal(big.reshape(20, 6144), alone_proofs[:20])
        st = srv.stats()
        assert st["requests"] == len(reqs) + 2 and st["p99_ms"] >= st["p50_ms"] > 0


def test_mix_equals_alone_digit_table_lanes():
    """Batches of up to 32 blobs: the lanes run the digit-table plan (chosen by
    the server's tuning) and share one table; every request's proofs equal the
    direct call's."""
    from conftest import random_blobs
    rng = np.random.default_rng(57)
    blobs = random_blobs(64, 1234)
    with vkzg_b200.Prover(max_batch_size=64) as p:
        alone = np.frombuffer(p.compute_cell_kzg_proofs_batch(blobs.tobytes(), 64), np.uint8).reshape(64, 6144)
    with vkzg_b200.Server(max_blobs_per_batch=32, lanes=2) as srv:
        reqs = []
        for _ in range(40):
            n = int(rng.integers(1, 9))
            s0 = int(rng.integers(0, 64 - n + 1))
            out = np.zeros(n * 6144, np.uint8)
            reqs.append((srv.submit_proofs(out, np.ascontiguousarray(blobs[s0:s0 + n]), n), s0, n, out))
        for t, s0, n, out in reqs:
            assert srv.wait(t) == 0
            assert np.array_equal(out.reshape(n, 6144), alone[s0:s0 + n]), (s0, n)
