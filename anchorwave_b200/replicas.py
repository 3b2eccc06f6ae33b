"""Replica sharding across GPUs (one process per GPU).

Interval pairs are independent, so a batch splits across ranks with no data-path
collective: each rank aligns its shard on its own GPU, and results are put back in the
caller's order.  Shards are balanced by longest-processing-time-first over the predicted DP
cells (qlen x tlen, or the band area), the load-balancing rule the reference's scheduler
uses for its cost-priority queue (src/service/AnchorTaskExecutor.h:54-160).
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def predicted_cells(qlen: int, tlen: int, band: int = -1) -> int:
    if band is None or band < 0 or band >= max(qlen, tlen):
        return qlen * tlen
    return (band + 1) * (qlen + tlen)


def lpt_shards(costs: Sequence[int], world: int) -> List[List[int]]:
    """Pair indices per rank; largest cost first onto the least-loaded rank (ties: lower rank)."""
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    for s in shards:
        s.sort()
    return shards


def merge_in_order(n: int, shards: Sequence[Sequence[int]], shard_results: Sequence[Sequence]) -> list:
    """Results of all shards back in the original pair order."""
    out = [None] * n
    for idx, res in zip(shards, shard_results):
        for i, r in zip(idx, res):
            out[i] = r
    return out
