"""Placement of independent systems on GPUs.

A population of realisations (the batched workload) needs no exchange
between systems, so ranks share them out and step their own subset with no
data-path collective; only the final per-system results are gathered.
Systems are placed longest-processing-time first by their O(N^2) pair-sum
cost, which keeps the ranks' work within one system of each other.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def lpt_partition(sizes: Sequence[int], ranks: int) -> List[List[int]]:
    """System indices per rank, placing the costliest (N^2) system first on
    the least-loaded rank; ties go to the lower rank, so the result is
    deterministic."""
    if ranks < 1:
        raise ValueError("ranks must be >= 1")
    order = sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]) ** 2, k))
    heap = [(0, r) for r in range(ranks)]
    heapq.heapify(heap)
    parts: List[List[int]] = [[] for _ in range(ranks)]
    for k in order:
        load, r = heapq.heappop(heap)
        parts[r].append(k)
        heapq.heappush(heap, (load + int(sizes[k]) ** 2, r))
    return [sorted(p) for p in parts]


def rank_share(sizes: Sequence[int], rank: int, world: int) -> List[int]:
    return lpt_partition(sizes, world)[rank]
