"""Multi-GPU plumbing of the explicit path (one process per GPU, torch.distributed).

The single-mesh benchmark runs replicas: every rank integrates its own copy of the mesh and
the ranks only agree on the timing (max over ranks) and the work done (sum over ranks). The
batched and served forms shard by solve: independent solves need no exchange, so each rank
takes a cost-balanced share (longest processing time first) and serves it on its own GPU.
No data-path collective exists on either path.
"""
from __future__ import annotations

import heapq


def reduce_max(value: float, dist=None, device: str = "cpu") -> float:
    """Max over ranks (a device time is the slowest rank's), or value alone without a group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(value: float, dist=None, device: str = "cpu") -> float:
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def aggregate_rate(work_local: float, seconds_local: float, dist=None, device: str = "cpu") -> float:
    """Whole-job throughput: the work of all ranks over the slowest rank's time."""
    return reduce_sum(work_local, dist, device) / reduce_max(seconds_local, dist, device)


def shard_by_cost(costs, world: int):
    """Indices of `costs` split into `world` shards of near-equal total cost (longest
    processing time first); every index lands in exactly one shard, each shard in input order."""
    heap = [(0.0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: -float(costs[k])):
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shards]


def request_cost(req) -> float:
    """Estimated device work of a solve: DOFs x RK steps."""
    _, _, nsteps = req.prepare()
    return float(req.ndofs) * nsteps
