"""Multi-GPU form of the EIP-7594 path: independent replicas.

Blobs are independent of one another in both vkzg_compute_proofs_batch and
vkzg_recover_cells_batch (vkzg.h: every output depends on one input blob), so
N GPUs split a batch into N contiguous shards and each rank runs its shard
through its own prover.  There is no exchange step on the data path; the only
cross-rank traffic is control: a barrier around timed regions, the maximum of
the per-rank times, and small result digests.  Works on any torch.distributed
backend (``gloo`` on CPU in the tests, ``nccl`` on GPUs).
"""


def shard_range(n_total, rank, world):
    """[lo, hi) of the blobs that `rank` of `world` owns: contiguous, sizes
    differing by at most one, earlier ranks taking the extra blobs."""
    if world < 1 or not 0 <= rank < world or n_total < 0:
        raise ValueError("bad shard request")
    base, extra = divmod(n_total, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def max_over_ranks(value, device=None):
    """Largest `value` over all ranks (the job's time is its slowest rank's)."""
    dist = _dist()
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(device=None):
    dist = _dist()
    if dist is not None:
        if device is not None and dist.get_backend() == "nccl":
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


def gather_outputs(local):
    """Every rank's output bytes, in rank order (a one-entry list without a
    group).  Concatenated, they are the whole batch's output in blob order,
    because shard_range() hands out contiguous shards in rank order."""
    dist = _dist()
    if dist is None:
        return [local]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, local)
    return out
