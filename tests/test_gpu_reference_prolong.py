"""Hierarchies built on the reference's own prolongation (chronos_amg_setup_prolong).

The reference keeps coarsening, C/F splitting and the prolongation on its host
code (cpt_aspAMG.m:224-225 calls prolong(...)) and forms the coarse operator
as Anext = Pf'*(A*Pf) (cpt_aspAMG.m:277).  Here every level's P comes from the
CPU path built with the reference's own FSAI and BAMG C++ (oracle/_ref); the
library computes the Galerkin products on the GPU, the FSAI factors, lambda_max
and omega, and the coarse factor.  Checked level by level against that CPU
path: level sizes equal, coarse operators with the same pattern bit for bit
and values within 1e-13 of the row's largest entry, FSAI factors with the same
pattern, omega within 5e-4 relative (eigs' tolerance in smoother.m:73-77), and
PCG_CJ iteration counts within one of the CPU path's.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import rowwise_close
import chronoslab_b200 as cb
from chronoslab_b200 import problems as PB
from oracle import amg_oracle as O

pytestmark = pytest.mark.gpu

# FP32 hierarchy (FP64 outer recurrence) against the FP64 CPU path: iterations
# within this many of its count.  The FP32 V-cycle is a slightly different
# preconditioner (values rounded to 24 bits), so one more iteration is allowed
# than for the FP64 hierarchy.
FP32_ITER_TOL = 2


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _reference(A, TV, b):
    from oracle import c_oracle as CO
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    H = CO.reference_hierarchy(A, TV, O.default_params())
    xo, ito, _, flo = CO.CHierarchy(H).pcg(b, itmax=1000, tol=1e-8)
    assert flo == 0
    return H, xo, ito


def _check_levels(h, H, value_tol):
    """Sizes, Galerkin operators, FSAI patterns and omega level by level."""
    assert h.nlevels == len(H.levels)
    for l, lv in enumerate(H.levels):
        Ag = h.export(l, "A")
        assert Ag.shape == lv.A.shape
        Ar = sp.csr_matrix(lv.A)
        Ar.sort_indices()
        # level 0 is the input; deeper levels are the GPU Galerkin products
        assert np.array_equal(Ag.indptr, Ar.indptr) and np.array_equal(Ag.indices, Ar.indices), l
        assert rowwise_close(Ag, Ar, value_tol), l
        if l == len(H.levels) - 1:
            break
        info = h.level_info(l)
        Gg = h.export(l, "G")
        Gr = sp.csr_matrix(lv.G)
        Gr.sort_indices()
        assert np.array_equal(Gg.indptr, Gr.indptr) and np.array_equal(Gg.indices, Gr.indices), l
        assert rowwise_close(Gg, Gr, 1e-8), l
        assert abs(info["lambda"] - lv.lam) <= 5e-4 * lv.lam, (l, info["lambda"], lv.lam)
        assert abs(info["omega"] - lv.omega) <= 5e-4 * lv.omega, (l, info["omega"], lv.omega)
        Pg = h.export(l, "P")
        assert (Pg != sp.csr_matrix(lv.P)).nnz == 0, l


def _solve_and_check(h, A, b, xo, ito, tol_it):
    x, it, _, flag, _ = h.pcg(b, itmax=1000, tol=1e-8)
    assert flag == 0
    assert abs(it - ito) <= tol_it, (it, ito)
    assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b)
    assert rel(x, xo) <= 1e-6
    return it


@pytest.fixture(scope="module")
def elast20():
    A, X = PB.elasticity_q1(20, return_coords=True)
    TV = PB.rbm_test_space(X)
    b = PB.elasticity_rhs(A, X, seed=0)
    H, xo, ito = _reference(A, TV, b)
    return A, b, H, xo, ito


@pytest.mark.parametrize("prec", [cb.CHRONOS_FP64, cb.CHRONOS_FP32])
def test_elasticity20_on_the_reference_prolongation(lib, elast20, prec):
    A, b, H, xo, ito = elast20
    Ps = [lv.P for lv in H.levels[:-1]]
    with cb.Hierarchy.with_prolongation(A, Ps, cb.params(precision=prec)) as h:
        _check_levels(h, H, 1e-13)
        _solve_and_check(h, A, b, xo, ito, 1 if prec == cb.CHRONOS_FP64 else FP32_ITER_TOL)


def test_prolongation_callback_sees_the_galerkin_operators(lib, elast20):
    """The callback form: it receives level l's operator (the GPU Galerkin
    product from level 2 on), equal in pattern to the CPU path's and in values
    to 1e-13, and returns that level's P."""
    A, b, H, xo, ito = elast20
    seen = []

    def prolong(level, Al):
        seen.append(level)
        Ar = sp.csr_matrix(H.levels[level - 1].A)
        Ar.sort_indices()
        assert np.array_equal(Al.indptr, Ar.indptr) and np.array_equal(Al.indices, Ar.indices)
        assert rowwise_close(Al, Ar, 1e-13)
        return H.levels[level - 1].P

    with cb.Hierarchy.with_prolongation(A, prolong, cb.params(precision=cb.CHRONOS_FP64)) as h:
        assert seen == list(range(1, len(H.levels)))
        _solve_and_check(h, A, b, xo, ito, 1)


def test_prolongation_callback_errors(lib):
    """A callback that raises or returns a P of the wrong shape fails the setup
    with an error and leaves no hierarchy behind."""
    A = PB.poisson7(12)
    held = cb.device_bytes()

    def boom(level, Al):
        raise ValueError("no prolongation here")

    with pytest.raises(ValueError):
        cb.Hierarchy.with_prolongation(A, boom, cb.params(ntv=1))
    with pytest.raises(cb.ChronosError):
        cb.Hierarchy.with_prolongation(A, [sp.identity(A.shape[0], format="csr")], cb.params(ntv=1))
    with pytest.raises(cb.ChronosError):
        P = sp.random(A.shape[0] - 1, 40, density=0.05, format="csr", random_state=0)
        cb.Hierarchy.with_prolongation(A, [P], cb.params(ntv=1))
    assert cb.device_bytes() == held


def test_c2_elasticity80_on_the_reference_prolongation(lib):
    """The C2 configuration at full size (Q1 elasticity 80^3, 1,574,640 DOF,
    rigid-body test space, BAMG, aFSAI; PCG_CJ to 1e-8 from x0 = 0) on the
    reference's own prolongation: level sizes equal, coarse operators with the
    CPU path's pattern bit for bit, iterations within one (FP64 hierarchy) and
    within FP32_ITER_TOL (FP32 hierarchy, FP64 outer) of the CPU path's."""
    A, X = PB.elasticity_q1(80, return_coords=True)
    TV = PB.rbm_test_space(X)
    b = PB.elasticity_rhs(A, X, seed=0)
    H, xo, ito = _reference(A, TV, b)
    Ps = [lv.P for lv in H.levels[:-1]]
    for prec in (cb.CHRONOS_FP64, cb.CHRONOS_FP32):
        with cb.Hierarchy.with_prolongation(A, Ps, cb.params(precision=prec)) as h:
            sizes = [h.level_info(l)["n"] for l in range(h.nlevels)]
            assert sizes == [lv.A.shape[0] for lv in H.levels]
            for l in range(1, h.nlevels):
                Ag = h.export(l, "A")
                Ar = sp.csr_matrix(H.levels[l].A)
                Ar.sort_indices()
                assert np.array_equal(Ag.indptr, Ar.indptr) and np.array_equal(Ag.indices, Ar.indices)
                assert rowwise_close(Ag, Ar, 1e-13)
            for l in range(h.nlevels - 1):
                lv = H.levels[l]
                info = h.level_info(l)
                assert abs(info["lambda"] - lv.lam) <= 5e-4 * lv.lam, (l, info["lambda"], lv.lam)
                assert abs(info["omega"] - lv.omega) <= 5e-4 * lv.omega
            _solve_and_check(h, A, b, xo, ito, 1 if prec == cb.CHRONOS_FP64 else FP32_ITER_TOL)
