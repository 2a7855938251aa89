"""Scene sharding across GPUs for the batched / serving forms.

Independent scenes partition with no exchange on the data path: each rank
steps its own scenes in one batched state, and only per-rank timings and
results travel between processes (torch.distributed, NCCL on GPUs, gloo on
CPU).  The partition is the longest-processing-time greedy rule on each
scene's particle-steps, so ranks get near-equal work; every rank computes the
same partition from the same sizes.
"""
from __future__ import annotations

import heapq


def shard_scenes(work, world: int) -> list[list[int]]:
    """Scene indices per rank, greedy by decreasing ``work[i]`` (ties by index)."""
    heap = [(0.0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for i in sorted(range(len(work)), key=lambda k: (-work[k], k)):
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(work[i]), r))
    return [sorted(s) for s in shards]


def all_max(x: float, world: int, device: str = "cuda") -> float:
    """Maximum of ``x`` over the ranks of the default process group."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def all_sum(x: float, world: int, device: str = "cuda") -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
