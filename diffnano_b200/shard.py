"""Work split across GPUs for the independent units of the path.

The FDTD path has no exchange step between units: batched instances,
wavelength sweeps, erosion/dilation variants, finite-difference probes and
prescreen candidates are independent.  With one process per GPU each rank
takes a share of the units, balanced by estimated cost (cells x steps), and
runs it alone; the only cross-rank traffic is the timing (max over ranks) and,
where a caller wants everything on one rank, gathering small results.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def shard_by_cost(costs: Sequence[float], world: int) -> List[List[int]]:
    """Indices of ``costs`` for each of ``world`` ranks: greedy longest-first
    assignment to the least-loaded rank (deterministic: ties go to the lower
    rank, equal costs keep their order).  Every index appears exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shards]


def rank_share(costs: Sequence[float], world: int, rank: int) -> List[int]:
    """This rank's indices (see :func:`shard_by_cost`)."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside [0, {world})")
    return shard_by_cost(costs, world)[rank]


def max_over_ranks(x: float, world: int, device=None) -> float:
    """The largest ``x`` over all ranks (timing); ``x`` itself when world is 1."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int, device=None) -> float:
    """Sum of ``x`` over all ranks (work counts)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
