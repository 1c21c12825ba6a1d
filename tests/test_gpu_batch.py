"""Batch of independent problems of uneven sizes (Poisson and log-normal
diffusion): every problem of the batch solve returns what its own
single-problem solve returns."""
import numpy as np
import pytest

import chronoslab_b200 as cb
from chronoslab_b200 import problems as PB

pytestmark = pytest.mark.gpu


def make_problems(seed, count):
    rng = np.random.default_rng(seed)
    As, bs = [], []
    for p in range(count):
        e = int(rng.integers(8, 25))
        if p % 2 == 0:
            A = PB.poisson7(e)
        else:
            A, _ = PB.diffusion7(e, sigma=2.0, corr_len=4.0, zaniso=0.01, seed=100 + p)
        As.append(A)
        bs.append(PB.uniform_rhs(A.shape[0], seed=200 + p))
    return As, bs


@pytest.mark.parametrize("prec", [cb.CHRONOS_FP32, cb.CHRONOS_FP64])
def test_batch_matches_single_solves(lib, prec):
    As, bs = make_problems(3, 7)
    bs[4] = np.zeros_like(bs[4])              # a zero right-hand side in the batch
    prm = cb.params(precision=prec, ntv=1)
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
            assert its[p] == it and flag == 0
            assert np.allclose(xs[p], x, rtol=1e-12, atol=1e-14 * np.abs(x).max())
            assert np.linalg.norm(b - A @ xs[p]) <= 1e-8 * np.linalg.norm(b)
        # repeated solves on the same batch
        xs2, its2, _, _ = B.solve(bs, itmax=1000, tol=1e-8)
        assert np.array_equal(its, its2)
        assert all(np.array_equal(a, c) for a, c in zip(xs, xs2))
