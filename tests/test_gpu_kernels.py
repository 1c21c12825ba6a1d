"""GPU parity of the individual kernels against the oracle / golden vectors,
all through the C ABI."""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import rowwise_close
import chronoslab_b200 as cb
from chronoslab_b200 import problems as PB

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("precision,tol", [(cb.CHRONOS_FP64, 1e-14), (cb.CHRONOS_FP32, 2e-6)])
def test_spmv_cubo(lib, cubo, precision, tol):
    A = cubo["Af"]
    x = np.random.default_rng(0).uniform(-1, 1, A.shape[0])
    y = cb.spmv(A, x, precision)
    ref = A @ x
    if precision == cb.CHRONOS_FP32:
        ref = (A.astype(np.float32) @ x.astype(np.float32)).astype(np.float64)
    assert rel(y, ref) <= tol


@pytest.mark.parametrize("precision,tol", [(cb.CHRONOS_FP64, 1e-14), (cb.CHRONOS_FP32, 2e-6)])
def test_spmv_shapes(lib, precision, tol):
    rng = np.random.default_rng(1)
    for A in (PB.poisson7(12), PB.elasticity_q1(5), sp.random(500, 300, 0.05, random_state=2,
                                                              format="csr")):
        x = rng.uniform(-1, 1, A.shape[1])
        y = cb.spmv(A, x, precision)
        assert rel(y, A @ x) <= max(tol, 1e-6 if precision == cb.CHRONOS_FP32 else tol)


def test_spmv_empty_rows(lib):
    A = sp.csr_matrix(([2.0, 3.0], ([0, 3], [1, 2])), shape=(5, 4))
    y = cb.spmv(A, np.arange(4.0))
    assert np.array_equal(y, A @ np.arange(4.0))


def test_fsai_numeric_vs_reference(lib, cubo, cubo_ref):
    """GPU local solves on the reference's own pattern reproduce its values."""
    Gref = cubo_ref["G"]
    vals, ok = cb.fsai_numeric(cubo["Af"], Gref)
    assert ok
    assert rowwise_close(Gref.__class__((vals, Gref.indices, Gref.indptr), shape=Gref.shape), Gref, 1e-10)


def test_fsai_drop_in_vs_reference(lib, cubo, cubo_ref):
    """SYM_aFSAI_compute mirror: host pattern + GPU values == reference MEX output."""
    F, ok = cb.afsai_cpp(cubo["Af"], 8, 15, 1, 1e-3)
    Gref = cubo_ref["G"]
    assert ok
    assert np.array_equal(F.indptr, Gref.indptr)
    assert np.array_equal(F.indices, Gref.indices)
    assert rowwise_close(F, Gref, 1e-10)


def test_fsai_small_reference(lib, small_ref):
    for A, G in ((small_ref["Ap"], small_ref["Gp"]), (small_ref["Ae"], small_ref["Ge"])):
        F, ok = cb.afsai_cpp(A, 2, 15, 1, 1e-3)
        assert ok
        assert np.array_equal(F.indices, G.indices) and np.array_equal(F.indptr, G.indptr)
        assert rowwise_close(F, G, 1e-10)


def test_fsai_indefinite_flag(lib):
    A = PB.poisson7(4).tolil()
    A[5, 5] = -1.0
    F, ok = cb.afsai_cpp(A.tocsr(), 1, 15, 1, 1e-3)
    assert not ok and F is None


def _scipy_galerkin(A, P):
    AP = (A @ P).tocsr()
    AP.eliminate_zeros()
    Pt = P.T.tocsr()
    Pt.sort_indices()
    Ac = (Pt @ AP).tocsr()
    Ac.eliminate_zeros()
    Ac.sort_indices()
    return Ac


def test_galerkin_bitexact_cubo(lib, cubo, cubo_ref):
    """Pattern and values bit-identical to a row-wise Gustavson P'(AP)."""
    A, P = cubo["Af"], cubo_ref["P"]
    Ac = cb.galerkin(A, P)
    ref = _scipy_galerkin(A, P)
    assert Ac.shape == ref.shape
    assert np.array_equal(Ac.indptr, ref.indptr)
    assert np.array_equal(Ac.indices, ref.indices)
    assert np.array_equal(Ac.data, ref.data)


def test_galerkin_bitexact_device_transpose(lib):
    """A prolongation of 2M entries: P' is built on the device (stable radix
    sort by column) and the 16-bit column offsets of A and P there too; the
    product is still bit-identical to the row-wise Gustavson one."""
    A = PB.poisson7(100)
    n = A.shape[0]
    nc = n // 8
    rng = np.random.default_rng(17)
    rows = np.repeat(np.arange(n), 2)
    cols = np.stack([np.arange(n) // 8, (np.arange(n) // 8 + 1 + np.arange(n) % 5) % nc], 1).ravel()
    P = sp.csr_matrix((rng.uniform(0.1, 1.0, 2 * n), (rows, cols)), shape=(n, nc))
    P.sum_duplicates()
    P.sort_indices()
    assert P.nnz >= 1 << 20
    Ac = cb.galerkin(A, P)
    ref = _scipy_galerkin(A, P)
    assert np.array_equal(Ac.indptr, ref.indptr)
    assert np.array_equal(Ac.indices, ref.indices)
    assert np.array_equal(Ac.data, ref.data)


def test_galerkin_cancellation_drops_zeros(lib):
    """Exact cancellations are dropped from the pattern, as MATLAB does."""
    A = PB.poisson7(6)
    n = A.shape[0]
    # piecewise-constant aggregation: row sums of A*P cancel exactly in the interior
    agg = np.arange(n) // 8
    P = sp.csr_matrix((np.ones(n), (np.arange(n), agg)), shape=(n, agg.max() + 1))
    Ac = cb.galerkin(A, P)
    ref = _scipy_galerkin(A, P)
    assert np.array_equal(Ac.indptr, ref.indptr) and np.array_equal(Ac.indices, ref.indices)
    assert np.array_equal(Ac.data, ref.data)
    assert np.all(Ac.data != 0)


def test_dense_chol(lib):
    rng = np.random.default_rng(3)
    for n in (1, 7, 64, 333):
        M = rng.standard_normal((n, n))
        A = M @ M.T + n * np.eye(n)
        L = cb.dense_chol(A)
        assert np.allclose(np.triu(L, 1), 0)
        assert np.linalg.norm(L - np.linalg.cholesky(A)) <= 1e-12 * np.linalg.norm(L)


def test_dense_chol_not_spd(lib):
    A = np.diag([1.0, 2.0, -3.0, 4.0])
    with pytest.raises(cb.ChronosError) as e:
        cb.dense_chol(A)
    assert e.value.code == -4


def mixed_rows(n=3000, ncols=2500, seed=7):
    """Mostly 3 entries per row, every 41st row 150-400 entries (the long-row
    path of every group width), every 97th row empty; columns spread so
    some rows need 32-bit columns and the rest 16-bit offsets."""
    rng = np.random.default_rng(seed)
    rows, cols = [], []
    for i in range(n):
        if i % 97 == 5:
            continue
        m = int(rng.integers(150, 400)) if i % 41 == 3 else 3
        c = rng.choice(ncols, size=m, replace=False)
        rows += [i] * m
        cols += c.tolist()
    vals = rng.uniform(-1, 1, len(rows))
    A = sp.csr_matrix((vals, (rows, cols)), shape=(n, ncols))
    A.sort_indices()
    return A


@pytest.mark.parametrize("ncols", [2500, 100000])          # 16-bit offsets / int32 columns
@pytest.mark.parametrize("precision", [cb.CHRONOS_FP64, cb.CHRONOS_FP32])
@pytest.mark.parametrize("fmt,lanes", [(1, 1), (1, 2), (1, 4), (1, 8), (1, 16), (1, 32), (2, 0),
                                       (0, 0)])
def test_apply_kernels_long_rows(lib, precision, fmt, lanes, ncols):
    """Every group width of the row-grouped CSR kernel and the sliced ELL
    kernel, with long rows (warp path), empty rows, and column spans that fit
    16-bit offsets or need int32 columns."""
    A = mixed_rows(ncols=ncols)
    x = np.random.default_rng(1).uniform(-1, 1, A.shape[1])
    y = cb.spmv(A, x, precision, format=fmt, lanes=lanes)
    if precision == cb.CHRONOS_FP32:
        ref = (A.astype(np.float32) @ x.astype(np.float32)).astype(np.float64)
        assert rel(y, ref) <= 2e-6
    else:
        assert rel(y, A @ x) <= 1e-14
    assert np.all(y[5::97] == 0.0)
