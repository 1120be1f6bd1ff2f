"""Pair-parallel registration across GPUs: one process per GPU, independent image pairs.

A set of registration pairs of uneven sizes is split across ranks by longest-processing-time
greedy bin packing on the per-pair cost (texels x control points in support), each rank
registers its own pairs on its own GPU with no collective on the data path, and the small
per-pair results are gathered at the end (one all_gather of Python objects).  Every rank
computes the same assignment from the same inputs, so no coordination is needed before the
work starts.
"""
from __future__ import annotations

import heapq
from typing import Callable, Dict, List, Sequence


def pair_cost(size, cp_spacing_voxels=4.0, support_voxels=12.0, D=3):
    """Work estimate of one optimizer iteration: texels x control points inside the support."""
    n = 1
    for s in size:
        n *= int(s)
    taps = (2.0 * support_voxels / cp_spacing_voxels) ** D
    return float(n) * taps


def assign_pairs(costs: Sequence[float], world: int) -> List[List[int]]:
    """LPT greedy: pairs in decreasing cost, each to the currently least-loaded rank.

    Deterministic (ties broken by pair index, then rank); returns the pair indices per rank.
    """
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(v) for v in out]


def imbalance(costs: Sequence[float], assignment: List[List[int]]) -> float:
    """max rank load / mean rank load (1.0 = perfect balance)."""
    loads = [sum(float(costs[i]) for i in a) for a in assignment]
    mean = sum(loads) / max(len(loads), 1)
    return max(loads) / mean if mean > 0 else 1.0


def run_pairs(costs: Sequence[float], register: Callable[[int], Dict], rank: int, world: int,
              group=None) -> List[Dict]:
    """Runs `register(pair_index)` for this rank's pairs and gathers all results on every rank.

    `register` returns a small dict (final value, iterations, seconds, ...).  With world == 1
    no process group is needed.
    """
    mine = assign_pairs(costs, world)[rank]
    local = [dict(register(i), pair=i, rank=rank) for i in mine]
    if world == 1:
        return local
    import torch.distributed as dist
    gathered: List[List[Dict]] = [None] * world  # type: ignore[list-item]
    dist.all_gather_object(gathered, local, group=group)
    out = [r for part in gathered for r in part]
    return sorted(out, key=lambda r: r["pair"])
