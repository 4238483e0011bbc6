"""Independent-unit sharding of band solves over ranks (one GPU per rank).

A band solve of one (cell, k-point) pair shares nothing with another, so many
of them (the k-points of a cell, the requests of a stream) spread over GPUs
with no collective on the data path: each rank solves whole units in its own
HBM, and only the eigenvalue vectors are gathered at the end (one
all-gather).  Inside one solve nothing is split.

Units go to ranks by longest-processing-time-first on an estimated cost
nb^2 * npw (the dense subspace and GEMM work) + nb * N log2 N (the FFTs), which
keeps the ranks' totals within one unit's cost of each other.  The assignment
depends only on the costs and the rank count, so every rank computes the same
one without communicating.
"""
from __future__ import annotations

import math
from typing import Callable, List, Sequence

import numpy as np


def unit_cost(npw: int, nbands: int, grid: Sequence[int]) -> float:
    """Estimated relative cost of one band solve."""
    n = int(np.prod(grid))
    return float(nbands) ** 2 * npw + float(nbands) * n * math.log2(max(n, 2))


def assign_units(costs: Sequence[float], world: int) -> List[List[int]]:
    """Partition unit indices over `world` ranks, largest first onto the least
    loaded rank (ties to the lower rank); each rank's list is in unit order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += costs[i]
    for lst in out:
        lst.sort()
    return out


def solve_sharded(units: Sequence, costs: Sequence[float], solve: Callable[[object], np.ndarray],
                  nbands: int, group=None) -> np.ndarray:
    """Solve the units assigned to this rank with `solve(unit) -> eigenvalues`
    and all-gather every unit's eigenvalues (shape (len(units), nbands)) onto
    every rank.  `group` is a torch.distributed process group (None: the
    default group, or a single process when torch.distributed is not
    initialised)."""
    import torch
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        world, rank = dist.get_world_size(group), dist.get_rank(group)
    else:
        world, rank = 1, 0
    mine = assign_units(costs, world)[rank]
    local = np.zeros((len(units), nbands), dtype=np.float64)
    for i in mine:
        local[i] = np.asarray(solve(units[i]), dtype=np.float64)[:nbands]
    if world == 1:
        return local
    # every unit is solved on exactly one rank and is zero elsewhere, so a sum
    # over ranks is the gather; the tensor lives where the backend wants it
    dev = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    t = torch.from_numpy(local).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()
