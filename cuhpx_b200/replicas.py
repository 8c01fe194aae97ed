"""Replicas over several GPUs (one process per GPU, torch.distributed).

Maps are independent, so a batch shards over ranks with no collective on the
data path: each rank transforms ``local_shard(x)`` with its own plans.  The
collectives here are only the bookkeeping around that: ``max_over_ranks``
(the timing rule: the slowest rank's time) and, when a caller wants every
rank to hold the whole result, ``gather_shards`` (one all_gather of the
shards, padded to the largest).  They work with any backend the process group
was created with (NCCL on the GPU, gloo on the CPU).
"""

import torch
import torch.distributed as dist


def _rank_world(rank, world):
    if rank is None or world is None:
        if dist.is_available() and dist.is_initialized():
            return dist.get_rank(), dist.get_world_size()
        return 0, 1
    return int(rank), int(world)


def shard_range(n, rank=None, world=None):
    """Contiguous [start, stop) of n items for this rank; sizes differ by at most one."""
    rank, world = _rank_world(rank, world)
    base, extra = divmod(int(n), world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def local_shard(x, rank=None, world=None):
    """This rank's slice of a batch along dim 0 (a view)."""
    start, stop = shard_range(x.shape[0], rank, world)
    return x[start:stop]


def max_over_ranks(value, device=None):
    """Max of a float over the ranks of the default group (the value itself without one)."""
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_shards(y, n_total):
    """All ranks' shards (dim 0, as shard_range splits n_total) concatenated in rank order."""
    if not (dist.is_available() and dist.is_initialized()):
        return y
    world = dist.get_world_size()
    size = max(shard_range(n_total, r, world)[1] - shard_range(n_total, r, world)[0] for r in range(world))
    pad = torch.zeros((size,) + tuple(y.shape[1:]), dtype=y.dtype, device=y.device)
    pad[: y.shape[0]] = y
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad)
    out = []
    for r in range(world):
        a, b = shard_range(n_total, r, world)
        out.append(parts[r][: b - a])
    return torch.cat(out, 0)
