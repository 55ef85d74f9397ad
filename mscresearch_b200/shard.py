"""Multi-GPU query sharding: one process per GPU, a replica of the graph on
each, queries dealt across ranks, answers gathered on every rank.

Queries are independent, so the only inter-rank traffic is the final
all-gather of the int64 answers (torch.distributed, NCCL on GPUs or gloo on
CPU).  The reference has no multi-GPU code (one hard-wired device,
Region_Aware_PR_with_Pruning_BoundaryCore.cu:2573).
"""
import numpy as np


def shard_bounds(nq, rank, world):
    """Contiguous balanced range [lo, hi) of the nq queries owned by rank."""
    base, extra = divmod(nq, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def solve_sharded(solve_fn, s, t, rank=None, world=None, device=None):
    """Solve queries (s[i], t[i]) spread over the ranks of the default process
    group.  solve_fn(s_part, t_part) -> int64 flows for that part (normally
    Graph.solve_batch bound to this rank's graph replica).  Returns all nq
    flows, in input order, on every rank."""
    import torch
    import torch.distributed as dist
    if world is None:
        world = dist.get_world_size() if dist.is_initialized() else 1
        rank = dist.get_rank() if dist.is_initialized() else 0
    s = np.asarray(s, np.int32)
    t = np.asarray(t, np.int32)
    nq = len(s)
    lo, hi = shard_bounds(nq, rank, world)
    local = np.asarray(solve_fn(s[lo:hi], t[lo:hi]), dtype=np.int64)
    if world == 1:
        return local
    width = shard_bounds(nq, 0, world)[1]  # the largest shard
    buf = torch.zeros(width, dtype=torch.int64, device=device)
    buf[: hi - lo] = torch.from_numpy(local).to(buf.device)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    out = np.empty(nq, np.int64)
    for r in range(world):
        a, b = shard_bounds(nq, r, world)
        out[a:b] = parts[r][: b - a].cpu().numpy()
    return out
