"""Right-preconditioned GMRES with the V-cycle (gmres_RIGHT.m) on the GPU,
against the oracle's restatement on the GPU hierarchy's own level matrices,
through the C ABI."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import chronoslab_b200 as cb
from chronoslab_b200 import problems as PB
from oracle import amg_oracle as O

pytestmark = pytest.mark.gpu


def oracle_hierarchy(h):
    parts = []
    for l in range(h.nlevels):
        info = h.level_info(l)
        p = {"A": h.export(l, "A")}
        if l < h.nlevels - 1:
            p.update(G=h.export(l, "G"), P=h.export(l, "P"), omega=info["omega"])
        parts.append(p)
    return O.hierarchy_from_parts(parts)


def total(it, restart):
    return (it[0] - 1) * restart + it[1]


def test_cubo_gmres_as_reference_calls_it(lib, cubo):
    """Tests/CubeBAMG_EMIN.m:22-31 calls gmres_RIGHT(A, rhs, 50, 1e-6, 100/50,
    M): the same call on the BAMG/aFSAI hierarchy (Tests/parm_*) takes the
    oracle's iteration count within one and meets the tolerance on the
    explicit residual."""
    A, Af, TV0 = cubo["A"], cubo["Af"], cubo["TV0"]
    b = np.ones(A.shape[0])
    with cb.Hierarchy(Af, TV0, cb.params(precision=cb.CHRONOS_FP64)) as h:
        x, flag, rel, it, rv = h.gmres(b, restart=50, tol=1e-6, maxit=2, A=A)
        Ho = oracle_hierarchy(h)
    xo, flo, relo, ito, rvo = O.gmres_right(lambda v: A @ v, b, 50, 1e-6, 2,
                                            mfun=lambda r: O.amg_vcycle(Ho, r))
    assert flag == 0 and flo == 0
    assert abs(total(it, 50) - total(ito, 50)) <= 1
    assert np.linalg.norm(b - A @ x) <= 1e-6 * np.linalg.norm(b)
    assert rv.size == total(it, 50) + 1 and rv[0] == pytest.approx(np.linalg.norm(b))
    assert np.linalg.norm(x - xo) <= 1e-5 * np.linalg.norm(xo)


@pytest.mark.parametrize("prec", [cb.CHRONOS_FP64, cb.CHRONOS_FP32])
def test_restarted_elasticity(lib, prec):
    """GMRES(5) restarts several times; FP64 and FP32 hierarchies reach the
    tolerance on the explicit residual within two iterations of the oracle."""
    A, X = PB.elasticity_q1(8, return_coords=True)
    TV = PB.rbm_test_space(X)
    b = PB.elasticity_rhs(A, X, seed=2)
    with cb.Hierarchy(A, TV, cb.params(precision=prec)) as h:
        x, flag, rel, it, rv = h.gmres(b, restart=5, tol=1e-8, maxit=40)
        Ho = oracle_hierarchy(h)
    xo, flo, _, ito, _ = O.gmres_right(lambda v: A @ v, b, 5, 1e-8, 40,
                                       mfun=lambda r: O.amg_vcycle(Ho, r))
    assert flag == 0 and flo == 0 and it[0] > 1
    assert abs(total(it, 5) - total(ito, 5)) <= 2
    assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b)


def test_edges_and_not_converged(lib):
    """b = 0 gives x = 0 and iter [0 0]; a solved x0 returns at once; too few
    cycles give flag 1 with the minimal-residual iterate, as the oracle."""
    A = PB.poisson7(12)
    n = A.shape[0]
    b = PB.uniform_rhs(n, seed=5)
    with cb.Hierarchy(A, np.ones((n, 1)), cb.params(precision=cb.CHRONOS_FP64)) as h:
        x, flag, rel, it, rv = h.gmres(np.zeros(n), restart=10, tol=1e-8, maxit=3)
        assert flag == 0 and it == (0, 0) and rel == 0.0 and not x.any()
        xs = spla.spsolve(A.tocsc(), b)
        x, flag, rel, it, rv = h.gmres(b, restart=10, tol=1e-8, maxit=3, x0=xs)
        assert flag == 0 and it == (0, 0) and rv.size == 1
        x, flag, rel, it, rv = h.gmres(b, restart=2, tol=1e-14, maxit=2)
        Ho = oracle_hierarchy(h)
    xo, flo, relo, ito, rvo = O.gmres_right(lambda v: A @ v, b, 2, 1e-14, 2,
                                            mfun=lambda r: O.amg_vcycle(Ho, r))
    assert flag == 1 and flo == 1
    assert rv.size == rvo.size == 2 * 2 + 1
    assert it == ito
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)


def test_reference_named_wrapper(lib):
    """cb.gmres_RIGHT follows gmres_RIGHT.m's argument defaults: restarted
    GMRES(restart) for maxit cycles, or the unrestarted method for maxit
    iterations when restart is None."""
    A = PB.poisson7(10)
    n = A.shape[0]
    b = PB.uniform_rhs(n, seed=8)
    with cb.Hierarchy(A, np.ones((n, 1)), cb.params(precision=cb.CHRONOS_FP64)) as h:
        r1 = cb.gmres_RIGHT(h, b, 5, 1e-8, 20)
        r2 = h.gmres(b, restart=5, tol=1e-8, maxit=20)
        assert r1[1] == r2[1] == 0 and r1[3] == r2[3] and np.array_equal(r1[0], r2[0])
        x, flag, rel, it, rv = cb.gmres_RIGHT(h, b, None, 1e-8, 40)
        assert flag == 0 and it[0] == 1 and rel <= 1e-8
