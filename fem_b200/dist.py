"""Multi-GPU plumbing for independent cells ("replicas only").

Cells are independent (the reference fans 8 of them out over OpenMP threads,
SamplesGenerator/SamplesGeneratorImpl.cpp:3707-3719), so N GPUs split the
cells with no data-path collective; the only collective is the max over ranks
of the measured device time (one all-reduce), and an optional gather of the
results.
"""
from __future__ import annotations

from typing import Sequence


def shard(weights: Sequence[float], world: int) -> list[list[int]]:
    """Split cell indices over `world` ranks, balancing the summed weight
    (voxels x expected iterations).  Greedy longest-processing-time: cells in
    decreasing weight go to the currently lightest rank; deterministic."""
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += weights[i]
    return [sorted(o) for o in out]


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar over the default process group (1 all-reduce)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
