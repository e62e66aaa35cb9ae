"""Sharding a batch of independent pencils over GPUs (one process per GPU).

The pencils are independent, so the batch splits with no data-path
collective: each rank solves its share as one level-batched launch sequence
(``AmlsSolver.solve_batch``) and only the results are gathered.  The share
is the longest-processing-time-first assignment by DOF^3, the order in which
the dense work of a pencil (its separator factorisations and eigensolves)
grows.
"""
from __future__ import annotations

import heapq

import numpy as np


def lpt_assign(sizes, ranks: int) -> list[list[int]]:
    """Pencil indices per rank: largest cost (size^3) first, each to the
    currently least loaded rank (ties to the lower rank).  Every rank's list
    is in ascending pencil order."""
    if ranks < 1:
        raise ValueError("ranks must be >= 1")
    cost = np.asarray(sizes, dtype=np.float64) ** 3
    order = sorted(range(len(cost)), key=lambda i: (-cost[i], i))
    heap = [(0.0, r) for r in range(ranks)]
    out: list[list[int]] = [[] for _ in range(ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + cost[i], r))
    return [sorted(x) for x in out]


def gather_thetas(local: dict, rank: int, world: int, dist, count: int):
    """Collect {pencil index: theta} from every rank on rank 0, returned in
    pencil order there (None on the other ranks).  Every rank calls it."""
    if dist is None or world == 1:
        return [local[i] for i in range(count)]
    parts = [None] * world
    dist.all_gather_object(parts, local)
    if rank != 0:
        return None
    merged = {}
    for p in parts:
        merged.update(p)
    if sorted(merged) != list(range(count)):
        raise RuntimeError("gathered pencils do not cover the batch")
    return [merged[i] for i in range(count)]


def solve_sharded(solver, pencils, opt, rank: int, world: int, dist):
    """This rank's share of the batch in one solve_batch call, thetas
    gathered on rank 0 (pencil order)."""
    share = lpt_assign([p.n for p in pencils], world)[rank]
    local = {}
    if share:
        sols = solver.solve_batch([pencils[i].K for i in share], [pencils[i].M for i in share], opt)
        local = {i: s.theta for i, s in zip(share, sols)}
    return gather_thetas(local, rank, world, dist, len(pencils))
