"""Sharding of independent solve instances over ranks (one process per GPU).

A batch of independent Poisson instances (the batched uneven-level family) has no exchange step:
every rank solves its own subset with its own BatchPCG and only the per-instance results are
gathered at the end.  The subsets come from a greedy longest-processing-time assignment on the
instances' cost (DOF count): instances in decreasing cost order, each to the currently least loaded
rank (ties to the lower rank, equal costs in index order), so every rank computes the same
partition without communicating.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def lpt_partition(costs: Sequence[float], parts: int) -> List[List[int]]:
    """Instance indices per part (each list ascending); deterministic."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, p) for p in range(parts)]
    heapq.heapify(heap)
    out: List[List[int]] = [[] for _ in range(parts)]
    for i in order:
        load, p = heapq.heappop(heap)
        out[p].append(i)
        heapq.heappush(heap, (load + float(costs[i]), p))
    return [sorted(o) for o in out]


def shard(costs: Sequence[float], rank: int, world: int) -> List[int]:
    """The instances rank `rank` of `world` solves."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return lpt_partition(costs, world)[rank]


def loads(costs: Sequence[float], parts: List[List[int]]) -> List[float]:
    return [float(sum(costs[i] for i in p)) for p in parts]


def gather_results(pg, rank: int, world: int, mine: List[int], values: Sequence[float], n: int) -> List[float]:
    """All ranks' per-instance values (e.g. iteration counts or final defects) in instance order,
    from each rank's own (indices, values); `pg` is torch.distributed (any backend with
    all_gather_object) or None for one rank."""
    if len(mine) != len(values):
        raise ValueError("one value per owned instance")
    out = [float("nan")] * n
    if pg is None or world == 1:
        for i, v in zip(mine, values):
            out[i] = float(v)
        return out
    parts = [None] * world
    pg.all_gather_object(parts, (list(mine), [float(v) for v in values]))
    seen = set()
    for idx, vals in parts:
        for i, v in zip(idx, vals):
            if i in seen:
                raise RuntimeError(f"instance {i} solved by two ranks")
            seen.add(i)
            out[i] = v
    if len(seen) != n:
        raise RuntimeError("instances missing from the gather")
    return out
