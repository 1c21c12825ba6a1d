"""Multi-GPU plumbing for batches of independent problems and blocks of
right-hand sides (one process per GPU, torch.distributed).

A single solve does not shard (dependent SpMVs, global dot products), so N
GPUs either run N replicas or split independent units:

* a batch of independent problems (ShardedBatch): problems are assigned
  largest-first to the least-loaded rank (weight = stored entries of the
  level-1 operator); each rank sets up and solves only its share;
* a block of right-hand sides (ShardedBlock): each rank holds the hierarchy of
  the shared operator and solves a contiguous share of the columns.

There is no collective on the data path: each rank's solve touches only its
own GPU, and the per-unit results (solutions if asked for, iterations, flags)
and the per-rank device times are gathered once at the end.  The solver of a
rank's share is injectable (make_batch / make_block), so the same plumbing
runs the GPU library in production and a CPU solver in tests.
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


def split_columns(ncols, nranks):
    """Contiguous column ranges [lo, hi) per rank, sizes differing by at most one."""
    base, extra = divmod(ncols, nranks)
    out, lo = [], 0
    for r in range(nranks):
        hi = lo + base + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def gather_results(local, world, dist):
    """All-gather of per-rank result dicts {unit index: value}; returns the
    merged dict on every rank (dist: torch.distributed or None)."""
    if world == 1 or dist is None:
        return dict(local)
    out = [None] * world
    dist.all_gather_object(out, local)
    merged = {}
    for d in out:
        merged.update(d)
    return merged


def _gather_times(seconds, world, rank, dist):
    return gather_results({rank: float(seconds)}, world, dist)


class ShardedBatch:
    """The rank's share of a batch of independent problems.

    As: every rank passes the whole list (the partition is computed the same
    way on every rank); only this rank's problems are set up.  make_batch(As)
    returns an object with solve(bs, itmax, tol) -> (xs, iters, flags,
    seconds); by default the GPU library's Batch with the given parameters.
    """

    def __init__(self, As, world=1, rank=0, dist=None, prm=None, make_batch=None):
        self.world, self.rank, self.dist = world, rank, dist
        self.parts = partition_largest_first([int(A.nnz) for A in As], world)
        self.mine = self.parts[rank]
        if make_batch is None:
            from . import Batch
            make_batch = lambda mats: Batch(mats, prm)  # noqa: E731
        self.local = make_batch([As[i] for i in self.mine]) if self.mine else None

    def solve_local(self, bs, itmax=1000, tol=1e-8):
        """This rank's problems only: (xs, iters, flags, seconds), in the
        order of self.mine."""
        if self.local is None:
            return [], [], [], 0.0
        return self.local.solve([bs[i] for i in self.mine], itmax=itmax, tol=tol)

    def solve(self, bs, itmax=1000, tol=1e-8, gather_x=True):
        """Solves this rank's share, then gathers the per-problem results.
        Returns ({problem: {"iters", "flag"[, "x"]}}, {rank: seconds}) on
        every rank; the batch's time is the slowest rank's."""
        xs, its, fls, sec = self.solve_local(bs, itmax, tol)
        local = {}
        for k, i in enumerate(self.mine):
            d = {"iters": int(its[k]), "flag": int(fls[k])}
            if gather_x:
                d["x"] = xs[k]
            local[i] = d
        return (gather_results(local, self.world, self.dist),
                _gather_times(sec, self.world, self.rank, self.dist))

    def close(self):
        if self.local is not None and hasattr(self.local, "close"):
            self.local.close()
        self.local = None


class ShardedBlock:
    """The rank's share of a block of right-hand sides of one operator.

    Every rank holds the operator's hierarchy (make_block(A) -> an object with
    pcg_block(B, itmax=, tol=) -> (X, iters, flags, seconds); by default the
    GPU library's Hierarchy with the constant test vector) and solves the
    columns split_columns assigns it.
    """

    def __init__(self, A, ncols, world=1, rank=0, dist=None, prm=None, make_block=None):
        self.world, self.rank, self.dist = world, rank, dist
        self.ranges = split_columns(ncols, world)
        self.lo, self.hi = self.ranges[rank]
        if make_block is None:
            import numpy as np
            from . import Hierarchy
            make_block = lambda M: Hierarchy(M, np.ones(M.shape[0]), prm)  # noqa: E731
        self.local = make_block(A) if self.hi > self.lo else None

    def solve_local(self, B, itmax=1000, tol=1e-8):
        if self.local is None:
            return None, [], [], 0.0
        return self.local.pcg_block(B[:, self.lo:self.hi], itmax=itmax, tol=tol)

    def solve(self, B, itmax=1000, tol=1e-8, gather_x=True):
        """Returns ({column: {"iters", "flag"[, "x"]}}, {rank: seconds})."""
        X, its, fls, sec = self.solve_local(B, itmax, tol)
        local = {}
        for k, j in enumerate(range(self.lo, self.hi)):
            d = {"iters": int(its[k]), "flag": int(fls[k])}
            if gather_x:
                d["x"] = X[:, k].copy()
            local[j] = d
        return (gather_results(local, self.world, self.dist),
                _gather_times(sec, self.world, self.rank, self.dist))

    def close(self):
        if self.local is not None and hasattr(self.local, "close"):
            self.local.close()
        self.local = None
