"""Multi-GPU plumbing of the query path (one process per GPU, torch.distributed).

Queries are independent and the mesh / cloud / scene structures are read-only, so the path shards
with no data-path collective: every rank holds a replica of the structure and evaluates its own
points.  The only collectives are the timing reduction (max over ranks) and barriers.
"""
from __future__ import annotations


def shard_range(n: int, rank: int, world: int):
    """Contiguous [begin, end) slice of n queries for `rank` of `world` (sizes differ by at most 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    base, extra = divmod(n, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks of the default process group (value itself without
    one).  `device`: where the reduction tensor lives (a CUDA device for NCCL, None = CPU/gloo)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
