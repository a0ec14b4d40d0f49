"""Multi-rank work split (one process per GPU, independent units): the
balanced partition, and the rank-level reductions the bench uses, run as two
gloo ranks on the CPU."""

from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from diffnano_b200.shard import max_over_ranks, rank_share, shard_by_cost, sum_over_ranks


def test_shard_partition_and_balance():
    g = torch.Generator().manual_seed(0)
    sides = torch.tensor([128, 192, 256, 384, 512, 768, 1024])[torch.randint(0, 7, (64,),
                                                                              generator=g)]
    costs = [float(s * s * (1500 + (s - 128) * 4500 / 896)) for s in sides]
    for world in (1, 2, 3, 4, 8):
        shards = shard_by_cost(costs, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(64))
        loads = [sum(costs[i] for i in s) for s in shards]
        # greedy longest-first: the heaviest rank exceeds the mean by at most one unit
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-6
        assert shards == shard_by_cost(costs, world)  # deterministic
    assert shard_by_cost([], 2) == [[], []]
    with pytest.raises(ValueError):
        shard_by_cost(costs, 0)
    with pytest.raises(ValueError):
        rank_share(costs, 2, 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = rank_share(costs, world, rank)
        work = sum(costs[i] for i in mine)
        total = sum_over_ranks(work, world)
        slowest = max_over_ranks(float(rank + 1), world)
        got = [None] * world
        dist.all_gather_object(got, mine)
        q.put((rank, got, total, slowest))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_and_reduce():
    costs = [float(c) for c in (5, 1, 9, 3, 3, 7, 2, 8)]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, total, slowest in out:
        assert sorted(i for s in got for i in s) == list(range(len(costs)))
        assert got == shard_by_cost(costs, world)
        assert total == sum(costs)
        assert slowest == float(world)
