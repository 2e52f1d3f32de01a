"""Splitting a batch of independent matrices across GPUs.

Batched factorizations need no communication: each GPU factors its own
matrices.  ``partition_by_cost`` assigns matrices to `parts` GPUs so that the
factorization work (n^3 / 3 each) is balanced: largest first, each to the
currently least-loaded part (the longest-processing-time rule).  Every rank
computes the same partition from the same sizes, so no exchange is needed.
"""
from __future__ import annotations

import heapq

import numpy as np


def partition_by_cost(sizes, parts: int) -> list[np.ndarray]:
    """Index arrays (ascending) of the matrices each of `parts` GPUs takes."""
    if parts <= 0:
        raise ValueError("parts must be positive")
    sizes = np.asarray(sizes, dtype=np.int64)
    order = np.argsort(-sizes, kind="stable")
    heap = [(0.0, p) for p in range(parts)]
    heapq.heapify(heap)
    bins = [[] for _ in range(parts)]
    for k in order:
        load, p = heapq.heappop(heap)
        bins[p].append(int(k))
        heapq.heappush(heap, (load + float(sizes[k]) ** 3 / 3.0, p))
    return [np.asarray(sorted(b), dtype=np.int64) for b in bins]


def shard_for_rank(sizes, rank: int, world: int) -> np.ndarray:
    """This rank's share of the batch (see partition_by_cost)."""
    return partition_by_cost(sizes, world)[rank]


def cost(sizes) -> float:
    return float(np.sum(np.asarray(sizes, dtype=np.float64) ** 3) / 3.0)
