"""Batched realizations split across ranks (one process per GPU).

Realizations of a Monte-Carlo batch are independent: no data of one enters
another's solve, so a batch shards by realization with no exchange on the
solve path.  Each rank solves the realizations assigned to it (one
``solve_batch`` launch sequence on its own GPU) and the per-realization
statistics are gathered afterwards, the only collective.

Assignment is longest-processing-time first: realizations in decreasing
order of estimated cost, each to the rank with the least cost so far (ties
to the lower rank), which bounds the slowest rank by 4/3 of the optimum.
The cost estimate is the number of (collocation point, source element)
pairs of one sweep, the dominant per-iteration work:
sum over element sides s of nint(s) * (elements of the side's fracture).
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def sweep_pairs(fractures: np.ndarray, elements: np.ndarray) -> int:
    """(collocation point, source) pairs of one sweep of a network."""
    nel = fractures["nelements"].astype(np.int64)
    ty = elements["_type"]
    nint = elements["nint"].astype(np.int64)
    keep = ty != 2  # wells have no collocation points
    total = int((nint[keep] * nel[elements["frac0"][keep]]).sum())
    inter = ty == 0
    total += int((nint[inter] * nel[elements["frac1"][inter]]).sum())
    return total


def partition_lpt(weights: Sequence[float], world_size: int) -> list[list[int]]:
    """Indices of the realizations each rank solves (longest processing time
    first); each rank's list is in increasing index order."""
    if world_size < 1:
        raise ValueError("world_size must be at least 1")
    w = np.asarray(weights, dtype=np.float64)
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    load = [0.0] * world_size
    parts: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += w[i]
    return [sorted(p) for p in parts]


def solve_batch_sharded(networks: Sequence, discharge_int: int, constants, *, rank: int | None = None,
                        world_size: int | None = None, solve_fn: Callable | None = None,
                        group=None) -> list[dict]:
    """Solves this rank's share of ``networks`` in place and returns the
    statistics of every realization (gathered from all ranks, in the order of
    ``networks``).  Only the records of this rank's share are updated.

    ``solve_fn(share, discharge_int, constants) -> list[dict]`` solves a list
    of (fractures, elements) pairs; the default is the GPU batch solve
    (``andfn_b200.solve_batch``).  Rank and world size default to those of the
    initialised torch.distributed process group (one rank when there is
    none)."""
    import torch.distributed as dist
    networks = list(networks)
    if rank is None or world_size is None:
        if dist.is_available() and dist.is_initialized():
            rank, world_size = dist.get_rank(group), dist.get_world_size(group)
        else:
            rank, world_size = 0, 1
    if solve_fn is None:
        from .batch import solve_batch as solve_fn
    parts = partition_lpt([sweep_pairs(F, E) for F, E in networks], world_size)
    mine = parts[rank]
    local = solve_fn([networks[i] for i in mine], discharge_int, constants) if mine else []
    if world_size == 1:
        return list(local)
    gathered: list = [None] * world_size
    dist.all_gather_object(gathered, list(zip(mine, local)), group=group)
    out: list = [None] * len(networks)
    for part in gathered:
        for i, st in part:
            out[i] = st
    return out
