"""Multi-GPU plumbing of the query path (one process per GPU, torch.distributed).

Queries are independent and the mesh / cloud / scene structures are read-only, so the path shards
with no data-path collective: every rank holds a replica of the structure and evaluates its own
contiguous slice of the points.  The optional exchange is an all-gather of the slices' results, so
that every rank holds the whole answer; the other collectives are the timing reduction (max over
ranks) and barriers.
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


def sharded_query(query, points, gather: bool = True):
    """Evaluates `query` (a callable taking a (m, 3) slice of `points` and returning a tensor whose
    first dimension is m, e.g. ``mesh.signed_distance``) on this rank's contiguous slice of
    `points`.  Without `gather`: returns (the slice's result, (begin, end)).  With `gather`: the
    slices' results are all-gathered over the default process group (NCCL over NVLink between
    GPUs; slices padded to equal length for the exchange), and every rank returns the full result
    for all of `points` with ((0, n)).  Outside an initialised process group it is one rank's
    whole query."""
    import torch
    import torch.distributed as dist
    n = int(points.shape[0])
    on = dist.is_available() and dist.is_initialized()
    rank, world = (dist.get_rank(), dist.get_world_size()) if on else (0, 1)
    begin, end = shard_range(n, rank, world)
    local = query(points[begin:end])
    if not gather or world == 1:
        return local, (begin, end)
    m = -(-n // world)
    padded = torch.zeros((m,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    padded[: end - begin] = local
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded)
    pieces = []
    for r in range(world):
        b, e = shard_range(n, r, world)
        pieces.append(parts[r][: e - b])
    return torch.cat(pieces), (0, n)
