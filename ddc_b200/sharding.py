"""Splitting the batch across GPUs: one process per GPU, each owning a share of the work.

Every batch line (and every problem of an uneven batch, and every field of a 2D build) is an
independent unit, so the path shards with no collective on the data path: each rank builds and
evaluates its own lines; the tiny plan (factor tables, knots) is created on every rank. The only
optional communication is gathering results on one rank when a caller wants them in one buffer.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def shard_range(n: int, rank: int, world: int) -> Tuple[int, int]:
    """[start, stop) of rank's contiguous share of n lines: sizes differ by at most one, lower
    ranks take the extra lines."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(n, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard_problems(costs: Sequence[float], world: int) -> List[List[int]]:
    """Problems of an uneven batch assigned to `world` ranks, largest first to the least loaded
    rank (the longest-processing-time rule); each rank's list keeps the problems' original order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    loads = [0.0] * world
    owner = [0] * len(costs)
    for i in sorted(range(len(costs)), key=lambda i: -costs[i]):
        r = min(range(world), key=lambda r: loads[r])
        owner[i] = r
        loads[r] += costs[i]
    return [[i for i in range(len(costs)) if owner[i] == r] for r in range(world)]


def problem_cost(ncells: int, degree: int, nevals: int) -> float:
    """Work estimate of one uneven-batch problem: rows swept times band width plus evaluated points
    times basis size."""
    return float(ncells) * (degree + 1) + float(nevals) * (degree + 1)
