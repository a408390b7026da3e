"""The multi-GPU form (independent replicas, vkzg_b200/replicas.py) on CPU: two
gloo ranks each take a shard of a batch, compute its cells and recover them
from half of the cells, and rank 0 checks that the gathered shards equal the
single-process result of the whole batch.  The per-shard work here is the
oracle standing in for each rank's GPU prover: what is under test is the
sharding, the gathering and the max-over-ranks timing, which have no GPU part.
"""
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from conftest import random_blobs
from vkzg_b200 import replicas

N_BLOBS = 3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _inputs():
    blobs = random_blobs(N_BLOBS, 77)
    present = np.zeros((N_BLOBS, 128), np.uint8)
    present[0, :64] = 1
    present[1, ::2] = 1
    present[2, np.random.default_rng(5).choice(128, 90, replace=False)] = 1
    return blobs, present


def _shard_work(lo, hi):
    from oracle import Oracle
    o = Oracle()
    blobs, present = _inputs()
    rc, cells = o.compute_cells(blobs[lo:hi], 1)
    assert rc == 0
    cells = np.asarray(cells, np.uint8).reshape(hi - lo, 128, 2048).copy()
    cells[present[lo:hi] == 0] = 0
    rc, rec = o.recover_cells(cells.reshape(hi - lo, -1), present[lo:hi], 1)
    assert rc == 0
    return np.asarray(rec, np.uint8).tobytes()


def _rank_main(rank, world, port, queue):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        lo, hi = replicas.shard_range(N_BLOBS, rank, world)
        out = _shard_work(lo, hi)
        replicas.barrier()
        parts = replicas.gather_outputs(out)
        slowest = replicas.max_over_ranks(10.0 + rank)
        if rank == 0:
            queue.put((b"".join(parts), slowest, [replicas.shard_range(N_BLOBS, r, world) for r in range(world)]))
    finally:
        dist.destroy_process_group()


def test_shard_range_covers_batch():
    for n in (0, 1, 2, 7, 256, 257):
        for world in (1, 2, 3, 8):
            spans = [replicas.shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.shard_range(4, 2, 2)


def test_no_group_is_identity():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.gather_outputs(b"abc") == [b"abc"]


def test_two_gloo_ranks_match_single_process():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        joined, slowest, spans = queue.get(timeout=300)
    finally:
        for p in procs:
            p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    assert spans == [(0, 2), (2, 3)]
    assert slowest == 11.0
    assert joined == _shard_work(0, N_BLOBS)
