"""Multi-GPU placement of independent MPM work (one process per GPU).

The substep has no exchange step between scenes, so work is spread over
ranks without any collective on the data path:

* a single scene runs as replicas (every rank advances its own copy);
* a batch of scenes is partitioned by particle count: largest scene first,
  each to the rank with the least work so far (greedy longest-processing-time),
  and every rank runs its share as one batched engine.

Only the measurement synchronises ranks: a barrier around the timed region
and the maximum of the per-rank device times.
"""
from __future__ import annotations

import os


def rank_info() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment."""
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def partition_scenes(sizes, world: int) -> list[list[int]]:
    """Scene indices for each of `world` ranks, balanced by particle count.

    Greedy longest-processing-time: scenes in decreasing size (ties by index)
    go to the rank with the smallest total so far (ties to the lowest rank);
    each rank's list is returned in ascending scene order.  Deterministic, so
    every rank computes the same partition without communicating."""
    if world < 1:
        raise ValueError("world size must be >= 1")
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(p) for p in parts]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of `value` over all ranks (the value itself without a process group)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    """The sum of `value` over all ranks (the value itself without a process group)."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
