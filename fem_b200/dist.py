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


def batch_sharded(engine, cells: Sequence, dLdC=None, weights: Sequence[float] | None = None,
                  allow_unconverged: bool = False, gather_grads: bool = True):
    """Independent cells over the ranks of the default process group: each rank
    solves its share (`shard`, weighted by voxels unless `weights` is given) in
    its own batched engine calls, then the results are gathered in cell order
    on every rank (one all-gather of host objects; no data-path collective).
    The reference's sample generator fans cells out over 8 OpenMP threads
    (SamplesGenerator/SamplesGeneratorImpl.cpp:3707-3719); here one rank per
    GPU takes that role.  Returns (C [n,6,6], infos, dL/drho list or None)
    like Engine.batch; every rank must call it with the same cells.  The
    gradients are one value per voxel (1.4 GB for the 4096-cell set):
    gather_grads=False keeps each rank's own (the other cells' entries are
    None)."""
    import numpy as np
    import torch.distributed as dist
    on = dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1
    world = dist.get_world_size() if on else 1
    rank = dist.get_rank() if on else 0
    w = list(weights) if weights is not None else [float(np.prod(c.shape)) for c in cells]
    mine = shard(w, world)[rank]
    dl = None if dLdC is None else np.asarray(dLdC, dtype=np.float64).reshape(len(cells), 6, 6)
    if mine:
        C, infos, grads = engine.batch([cells[i] for i in mine], dLdC=None if dl is None else dl[mine],
                                       allow_unconverged=allow_unconverged)
    else:
        C, infos, grads = np.zeros((0, 6, 6)), [], ([] if dl is not None else None)
    part = (mine, C, infos, grads if gather_grads else None)
    parts = [None] * world
    if on:
        dist.all_gather_object(parts, part)
    else:
        parts = [part]
    if not gather_grads and grads is not None:   # this rank's own gradients stay local
        parts[rank] = (mine, C, infos, grads)
    Cs = np.zeros((len(cells), 6, 6))
    all_infos = [None] * len(cells)
    all_grads = [None] * len(cells) if dl is not None else None
    for idx, Cp, ip, gp in parts:
        for k, i in enumerate(idx):
            Cs[i] = Cp[k]
            all_infos[i] = ip[k]
            if all_grads is not None and gp is not None:
                all_grads[i] = gp[k]
    return Cs, all_infos, all_grads
