"""Multi-GPU plumbing for batches of independent problems (one process per
GPU, torch.distributed).

A single solve does not shard (dependent SpMVs, global dot products), so N
GPUs either run N replicas or split a batch of independent problems: the
problems are assigned largest-first to the least-loaded rank (weight = stored
entries of the level-1 operator), each rank solves its share with no
collective on the data path, and the per-problem results (iterations, flags,
times) are gathered at the end.
"""
from __future__ import annotations

import heapq


def partition_largest_first(weights, nranks):
    """Greedy LPT assignment: returns a list of problem-index lists, one per
    rank, each in descending weight order."""
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    heap = [(0, r) for r in range(nranks)]
    heapq.heapify(heap)
    parts = [[] for _ in range(nranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + weights[i], r))
    return parts


def gather_results(local, world, dist):
    """All-gather of per-rank result dicts {problem index: value}; returns the
    merged dict on every rank (dist: torch.distributed or None)."""
    if world == 1 or dist is None:
        return dict(local)
    out = [None] * world
    dist.all_gather_object(out, local)
    merged = {}
    for d in out:
        merged.update(d)
    return merged
