"""Batch of independent problems of uneven sizes (Poisson and log-normal
diffusion): every problem of the batch solve returns what its own
single-problem solve returns."""
import numpy as np
import pytest

import chronoslab_b200 as cb
from chronoslab_b200 import problems as PB

pytestmark = pytest.mark.gpu


def make_problems(seed, count, lo=8):
    rng = np.random.default_rng(seed)
    As, bs = [], []
    for p in range(count):
        e = int(rng.integers(lo, 25))
        if p % 2 == 0:
            A = PB.poisson7(e)
        else:
            A, _ = PB.diffusion7(e, sigma=2.0, corr_len=4.0, zaniso=0.01, seed=100 + p)
        As.append(A)
        bs.append(PB.uniform_rhs(A.shape[0], seed=200 + p))
    return As, bs


@pytest.mark.parametrize("grouped", [0, 1])
@pytest.mark.parametrize("prec", [cb.CHRONOS_FP32, cb.CHRONOS_FP64])
def test_batch_matches_single_solves(lib, prec, grouped):
    """Per-stream mode: exactly the single solves.  Grouped mode (stacked
    level operators; G' stored times omega; FP64 outer operator): the single
    solves' iterations within 1 and their solutions to rounding level."""
    As, bs = make_problems(3, 7, lo=11 if grouped else 8)
    bs[4] = np.zeros_like(bs[4])              # a zero right-hand side in the batch
    prm = cb.params(precision=prec, ntv=1, batch_grouped=grouped)
    with cb.Batch(As, prm) as B:
        xs, its, fl, sec = B.solve(bs, itmax=1000, tol=1e-8)
        assert sec > 0
        for p, (A, b) in enumerate(zip(As, bs)):
            assert fl[p] == 0
            if p == 4:
                assert its[p] == 0 and not np.any(xs[p])
                continue
            with cb.Hierarchy(A, np.ones(A.shape[0]), cb.params(precision=prec, ntv=1)) as h:
                assert h.nlevels == B.nlevels(p)
                x, it, _, flag, _ = h.pcg(b, itmax=1000, tol=1e-8)
            assert flag == 0
            if grouped:
                assert abs(int(its[p]) - it) <= 1
                tol = 1e-6 if prec == cb.CHRONOS_FP32 else 1e-9
                assert np.linalg.norm(xs[p] - x) <= tol * np.linalg.norm(x)
            else:
                assert its[p] == it
                assert np.allclose(xs[p], x, rtol=1e-12, atol=1e-14 * np.abs(x).max())
            assert np.linalg.norm(b - A @ xs[p]) <= 1e-8 * np.linalg.norm(b)
        # repeated solves on the same batch
        xs2, its2, _, _ = B.solve(bs, itmax=1000, tol=1e-8)
        assert np.array_equal(its, its2)
        assert all(np.array_equal(a, c) for a, c in zip(xs, xs2))


def test_batch_grouped_with_single_level_problems(lib):
    """Problems small enough to be their own coarsest level: the batch falls
    back to one graph per problem and still matches the single solves."""
    As = [PB.poisson7(6), PB.poisson7(14), PB.poisson7(7)]
    bs = [PB.uniform_rhs(A.shape[0], seed=10 + p) for p, A in enumerate(As)]
    with cb.Batch(As, cb.params(ntv=1, batch_grouped=1)) as B:
        assert B.nlevels(0) == 1 and B.nlevels(1) >= 2
        xs, its, fl, _ = B.solve(bs, itmax=500, tol=1e-8)
        for A, b, x, f in zip(As, bs, xs, fl):
            assert f == 0
            assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b)


def test_batch_grouped_itmax_and_deep_mix(lib):
    """Problems of different depths in one grouped batch, and itmax reached:
    flag 1 for the problems that did not converge, iterations = itmax."""
    As, bs = make_problems(11, 6, lo=11)
    with cb.Batch(As, cb.params(ntv=1, batch_grouped=1)) as B:
        depths = {B.nlevels(p) for p in range(len(As))}
        xs, its, fl, _ = B.solve(bs, itmax=3, tol=1e-14)
        assert np.all(its == 3) and np.all(fl == 1)
        xs, its, fl, _ = B.solve(bs, itmax=1000, tol=1e-8)
        assert np.all(fl == 0)
        for A, b, x in zip(As, bs, xs):
            assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b)
    assert len(depths) >= 1


def test_batch_grouped_host_loop_matches_graph_loop(lib):
    """use_graph = 0 launches the grouped iteration from a host loop (what a
    profiler sees): the same results bit for bit."""
    As, bs = make_problems(5, 5, lo=11)
    out = []
    for g in (1, 0):
        with cb.Batch(As, cb.params(ntv=1, batch_grouped=1, use_graph=g)) as B:
            out.append(B.solve(bs, itmax=1000, tol=1e-8))
    assert np.array_equal(out[0][1], out[1][1])
    assert all(np.array_equal(a, c) for a, c in zip(out[0][0], out[1][0]))


def test_fsai_numeric_batch_bit_identical_for_every_tile_set(lib):
    """One batched FSAI numeric phase over several problems (local systems up
    to 60: FSAI 15 steps of 4) gives, for every candidate set of tile sizes
    and for the tuned one, each problem's values of chronos_fsai_numeric bit
    for bit; a batch of more than 20,000 rows is tuned."""
    As = [PB.poisson7(32), PB.diffusion7(14, sigma=2.0, corr_len=4.0, seed=3)[0],
          PB.elasticity_q1(6), PB.poisson7(9)]
    Gs = []
    for A in As:
        G, ok = cb.fsai_pattern(A, nstep=15, step_size=4, eps=1e-3, nthread=8)
        assert ok
        Gs.append(G)
    assert max(np.diff(G.indptr).max() for G in Gs) - 1 > 32
    want = [cb.fsai_numeric(A, G, base=0)[0] for A, G in zip(As, Gs)]
    for ts in (0, 1, 2, 3, -1):
        vals, oks, used = cb.fsai_numeric_batch(As, Gs, tile_set=ts)
        assert all(oks) and (used == ts if ts >= 0 else 0 <= used <= 3)
        for v, w in zip(vals, want):
            assert np.array_equal(v, w), ts


def test_batch_hierarchies_equal_single_builds(lib):
    """The level-synchronous batch setup (FSAI numeric batched across the
    problems) builds every problem's hierarchy as a single setup does: the
    same levels (the batched values themselves are checked bit for bit above,
    the solves against single ones in test_batch_matches_single_solves), and
    the batched numeric phase's time is attributed to the problems."""
    As, _ = make_problems(5, 6, lo=10)
    prm = cb.params(precision=cb.CHRONOS_FP64, ntv=1, nstep=15, step_size=4, batch_grouped=0)
    with cb.Batch(As, prm) as B:
        for p, A in enumerate(As):
            with cb.Hierarchy(A, np.ones(A.shape[0]), prm) as h:
                assert h.nlevels == B.nlevels(p)
        t = B.setup_times()
        assert t["fsai_numeric"] > 0.0
