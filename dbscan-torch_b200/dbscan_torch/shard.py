"""Partition independent clouds across ranks (one process per GPU).

The plain single-cloud path does not shard (a cloud would need a halo
exchange and a global renumbering of cluster ids), so multi-GPU runs of it
are replicas. Batched and served clouds are independent units: each rank
clusters its own subset with the batched pipeline, with no collective on the
data path. ``shard_clouds`` balances the subsets by work (points, the
quantity pipeline time and workspace scale with) with the longest-first
greedy rule: clouds in decreasing size, each to the currently lightest rank
(ties to the lower rank), which keeps every rank within the largest single
cloud of the mean load. The assignment depends only on the sizes, so every
rank computes the same one without communicating.
"""

from __future__ import annotations

import heapq
from typing import List, Sequence

import numpy as np


def shard_clouds(sizes: Sequence[int], world_size: int) -> List[List[int]]:
    """Cloud indices per rank (each list ascending)."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    sizes = np.asarray(sizes, dtype=np.int64)
    if (sizes < 0).any():
        raise ValueError("cloud sizes must be >= 0")
    order = np.lexsort((np.arange(sizes.size), -sizes))  # size descending, index ascending
    heap = [(0, r) for r in range(world_size)]
    out: List[List[int]] = [[] for _ in range(world_size)]
    for k in order.tolist():
        load, r = heapq.heappop(heap)
        out[r].append(k)
        heapq.heappush(heap, (load + int(sizes[k]), r))
    return [sorted(v) for v in out]


def shard_loads(sizes: Sequence[int], shards: List[List[int]]) -> List[int]:
    """Points per rank of an assignment."""
    sizes = np.asarray(sizes, dtype=np.int64)
    return [int(sizes[s].sum()) for s in shards]
