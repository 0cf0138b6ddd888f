"""Whole-system partition of a batch across GPUs (one process per GPU).

Independent systems need no exchange while they run, so a batch spread over several GPUs is a
set of smaller batches, one per rank, with no per-step collective: each rank creates a
`BatchSimulation` of the systems assigned to it and the results are gathered once at the end.
The assignment is the longest-processing-time rule: systems in decreasing order of estimated
cost, each to the rank with the least cost so far (ties to the lower rank), which keeps the
slowest rank within 4/3 of the best possible balance. It depends only on the costs and the
number of ranks, so every rank computes the same partition without communicating.
"""
from __future__ import annotations

import math
from typing import Sequence


def system_cost(atoms: int, box_volume_nm3: float, cutoff_nm: float, grid: Sequence[int]) -> float:
    """Estimated per-step work of one system: the pairs within the cutoff (the pair kernel's
    share, N * rho * (4/3) pi rc^3 / 2 at the system's atom density) plus the reciprocal grid's
    points weighted by the FFT's log2 length per axis (spreading, transforms and gather)."""
    if atoms <= 0:
        return 0.0
    density = atoms / box_volume_nm3
    pairs = 0.5 * atoms * density * (4.0 / 3.0) * math.pi * cutoff_nm ** 3
    points = float(grid[0]) * grid[1] * grid[2]
    fft = points * sum(math.log2(max(2, int(k))) for k in grid) / 3.0
    return pairs + fft


def partition_systems(costs: Sequence[float], ranks: int) -> list[list[int]]:
    """Assign system indices to `ranks` ranks (lists of indices, each in increasing order) by
    the longest-processing-time rule; a rank may get no system when there are fewer systems
    than ranks."""
    if ranks < 1:
        raise ValueError("ranks must be at least 1")
    if any(c < 0 or not math.isfinite(c) for c in costs):
        raise ValueError("costs must be finite and non-negative")
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    load = [0.0] * ranks
    parts: list[list[int]] = [[] for _ in range(ranks)]
    for k in order:
        r = min(range(ranks), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += costs[k]
    return [sorted(p) for p in parts]
