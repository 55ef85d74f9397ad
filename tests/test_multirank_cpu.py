"""World-size-2 gloo test of the query-sharding path (CPU, no GPU): each
rank solves its shard with the oracle standing in for its graph replica, and
the all-gathered answers must equal a single-process solve in input order."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mscresearch_b200.shard import shard_bounds


def test_shard_bounds_cover_exactly():
    for nq in (0, 1, 7, 256, 1001):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                lo, hi = shard_bounds(nq, r, world)
                seen += list(range(lo, hi))
            assert seen == list(range(nq))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from oracle import oracle as O
    from mscresearch_b200.shard import solve_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    rng = np.random.default_rng(3)
    n = 300
    u = rng.integers(0, n, 3000)
    v = rng.integers(0, n, 3000)
    c = rng.integers(1, 50, 3000)
    g = O.build_csr(n, u, v, c)
    s = rng.integers(0, n, 37)
    t = rng.integers(0, n, 37)
    flows = solve_sharded(lambda a, b: [O.dinic(g, x, y) for x, y in zip(a, b)], s, t)
    q.put((rank, list(flows), [O.dinic(g, x, y) for x, y in zip(s, t)]))
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_world2_sharded_equals_single():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, exp in res:
        assert got == exp
