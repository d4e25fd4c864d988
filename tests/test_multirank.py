"""The N > 1 paths on the CPU with world_size-2 gloo groups: the bench's max-over-ranks
timing and summed work, and the by-solve sharding of the batched / served forms."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from philip_b200.shard import aggregate_rate, reduce_max, shard_by_cost


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # replicas: rank r took (r + 1) ms for the same work
        ms = reduce_max(1.0 + rank, dist)
        rate = aggregate_rate(100.0, (1.0 + rank) * 1e-3, dist)
        # sharded solves: every rank derives the same shards and serves its own
        costs = [5, 1, 9, 3, 7, 2, 8, 4, 6, 10]
        mine = shard_by_cost(costs, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        out[rank] = (ms, rate, gathered)
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_and_sharding():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        ms, rate, gathered = res[r]
        assert ms == 2.0                           # the slowest rank's time
        assert abs(rate - 200.0 / 2e-3) < 1e-6     # all ranks' work over that time
        flat = sorted(i for s in gathered for i in s)
        assert flat == list(range(10))             # every solve exactly once
        assert gathered == res[0][2]               # same shards on every rank


def test_shard_balance():
    rng = np.random.default_rng(0)
    costs = rng.integers(1, 1000, size=200)
    shards = shard_by_cost(costs, 8)
    loads = [sum(costs[i] for i in s) for s in shards]
    assert max(loads) <= 1.05 * (sum(costs) / 8) + max(costs)
    assert sorted(i for s in shards for i in s) == list(range(200))
