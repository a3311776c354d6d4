"""Multi-process plumbing on CPU: two gloo ranks agree on the max-over-ranks step time and shard a
query set contiguously with nothing lost or duplicated."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from ebgeometry_b200.ranks import max_over_ranks, shard_range, sharded_query


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import torch
        ms = 10.0 + 5.0 * rank
        # a stand-in query (sum of coordinates, tagged with the rank that evaluated it) over a
        # point set that does not divide evenly: every rank ends with every point's answer
        pts = torch.arange(3 * 1001, dtype=torch.float64).reshape(1001, 3)
        full, span = sharded_query(lambda x: torch.stack([x.sum(1), torch.full((x.shape[0],), float(rank),
                                                                             dtype=torch.float64)], 1), pts)
        local, lspan = sharded_query(lambda x: x[:, 0], pts, gather=False)
        q.put((rank, max_over_ranks(ms), shard_range(1001, rank, world), full.numpy(), span, local.numpy(), lspan))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got.sort(key=lambda g: g[0])
    assert all(g[1] == 15.0 for g in got)
    spans = [g[2] for g in got]
    assert spans[0][0] == 0 and spans[-1][1] == 1001 and spans[0][1] == spans[1][0]
    import numpy as np
    pts = np.arange(3 * 1001, dtype=np.float64).reshape(1001, 3)
    for rank, _, _, full, span, local, lspan in got:
        assert span == (0, 1001) and full.shape == (1001, 2)
        assert np.array_equal(full[:, 0], pts.sum(1))
        # the first ceil(1001/2) answers came from rank 0, the rest from rank 1
        assert np.array_equal(full[:, 1], (np.arange(1001) >= spans[0][1]).astype(np.float64))
        assert lspan == spans[rank] and np.array_equal(local, pts[lspan[0]:lspan[1], 0])


@pytest.mark.parametrize("n,world", [(0, 3), (10, 4), (1000003, 8)])
def test_shard_range_partitions(n, world):
    spans = [shard_range(n, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == n
    assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
    sizes = [e - b for b, e in spans]
    assert max(sizes) - min(sizes) <= 1
