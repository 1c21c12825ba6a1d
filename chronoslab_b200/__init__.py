"""chronoslab_b200 -- B200-native (sm_100a) AMG-preconditioned SPD solve path of
ChronosLab, behind a C ABI (include/chronos_b200.h) with this Python binding.

The names mirror the reference's entry points on this path:
  cpt_aspAMG(param, A, TV0)            -> Hierarchy   (aspAMG/cpt_aspAMG.m)
  AMG_Vcycle(hrc, b)                   -> x           (aspAMG/AMG_Vcycle.m)
  PCG_CJ(hrc, b, x0, itmax, tol)       -> x, iter, resvec, flag   (LinearSolver/PCG_CJ.m)
  SQMR(hrc, rhs, tol, itmax)           -> x, info, relres, niter  (LinearSolver/SQMR.m)
  SYM_aFSAI_compute(...)               -> the MEX outputs         (MEX_SYM_AFSAI)
  afsai_cpp(M, nthread, nstep, step_size, eps) -> F, is_posdef    (smoother/afsai_cpp.m)
  readDefaultParams(fnames)            -> chronos_params          (utils/readDefaultParams.m)
Vectors are numpy FP64 arrays; matrices scipy.sparse CSR (0-based).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import scipy.sparse as sp

from ._lib import (CHRONOS_FP32, CHRONOS_FP64, ChronosError, chronos_level_info, chronos_params,
                   check, last_error, load)

__all__ = [
    "CHRONOS_FP32", "CHRONOS_FP64", "ChronosError", "Hierarchy", "Batch", "params",
    "readDefaultParams",
    "cpt_aspAMG", "AMG_Vcycle", "PCG_CJ", "SQMR", "SYM_aFSAI_compute", "afsai_cpp",
    "fsai_numeric", "fsai_pattern", "coarsen", "bamg", "emin_pattern", "emin", "galerkin",
    "dense_chol", "spmv",
    "diag_fix", "version",
]

_P_I = C.POINTER(C.c_int)
_P_I64 = C.POINTER(C.c_int64)
_P_D = C.POINTER(C.c_double)


def _pi(a):
    return a.ctypes.data_as(_P_I)


def _pi64(a):
    return a.ctypes.data_as(_P_I64)


def _pd(a):
    return a.ctypes.data_as(_P_D)


def version():
    return load().chronos_version().decode()


def _csr(A, ncols=None):
    A = sp.csr_matrix(A)
    if not A.has_sorted_indices:
        A = A.copy()
        A.sort_indices()
    indptr = np.ascontiguousarray(A.indptr, dtype=np.int32)
    indices = np.ascontiguousarray(A.indices, dtype=np.int32)
    data = np.ascontiguousarray(A.data, dtype=np.float64)
    return A.shape[0], indptr, indices, data


_STR_FIELDS = {"smoother_method", "tspace_method", "SoC_type", "proltype", "prol_emin",
               "rhs_build", "solv_method"}


def params(**overrides):
    """Reference regression-test defaults (Tests/parm_*), then overrides."""
    p = chronos_params()
    load().chronos_params_default(C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise KeyError(f"unknown parameter {k}")
        setattr(p, k, v.encode() if k in _STR_FIELDS else v)
    return p


def readDefaultParams(fnames_path, **overrides):
    """Reads aspAMG.fnames and the seven parm_* files it names."""
    p = params()
    check(load().chronos_params_read(str(fnames_path).encode(), C.byref(p)))
    for k, v in overrides.items():
        setattr(p, k, v.encode() if k in _STR_FIELDS else v)
    return p


class _CsrHandle:
    """Fetches a chronos_csr result into scipy and frees it."""

    @staticmethod
    def take(handle):
        lib = load()
        nr, nc, nnz = C.c_int(), C.c_int(), C.c_int64()
        check(lib.chronos_csr_info(handle, C.byref(nr), C.byref(nc), C.byref(nnz)))
        iat = np.zeros(nr.value + 1, np.int32)
        ja = np.zeros(max(nnz.value, 1), np.int32)
        v = np.zeros(max(nnz.value, 1), np.float64)
        check(lib.chronos_csr_fetch(handle, _pi(iat), _pi(ja), _pd(v)))
        check(lib.chronos_csr_free(handle))
        return sp.csr_matrix((v[:nnz.value], ja[:nnz.value], iat), shape=(nr.value, nc.value))


# ---------------------------------------------------------------------------
# FSAI
# ---------------------------------------------------------------------------

def SYM_aFSAI_compute(nthread, n_step, step_size, tau, eps, nrows, nrows_M, nterm_M, iat_M,
                      ja_M, coef_M):
    """Mirror of the MEX gateway SYM_aFSAI_compute.cpp:15-20: 1-based CSR with
    int64 iat / int32 ja; returns (nterm_G, iat_G, ja_G, coef_G, is_posdef)."""
    iat_M = np.ascontiguousarray(iat_M, dtype=np.int64)
    ja_M = np.ascontiguousarray(ja_M, dtype=np.int32)
    coef_M = np.ascontiguousarray(coef_M, dtype=np.float64)
    kmax = 1 + n_step * step_size
    iat_G = np.zeros(nrows + 1, np.int64)
    ja_G = np.zeros(nrows * kmax, np.int32)
    coef_G = np.zeros(nrows * kmax, np.float64)
    nterm = C.c_int64()
    posdef = C.c_int()
    check(load().chronos_fsai_compute(nthread, n_step, step_size, tau, eps, nrows, nrows_M,
                                      nterm_M, _pi64(iat_M), _pi(ja_M), _pd(coef_M),
                                      C.byref(nterm), _pi64(iat_G), _pi(ja_G), _pd(coef_G),
                                      C.byref(posdef)))
    nt = nterm.value
    return nt, iat_G, ja_G[:nt], coef_G[:nt], bool(posdef.value)


def afsai_cpp(M, nthread, nstep, step_size, eps):
    """afsai_cpp.m:1-65: F (lower-triangular CSR, diagonal last in each row)
    and is_posdef; F is None when the matrix was deemed indefinite."""
    M = sp.csr_matrix(M)
    M.sort_indices()
    n = M.shape[0]
    nt, iat, ja, coef, ok = SYM_aFSAI_compute(nthread, nstep, step_size, 0.0, eps, n, n, M.nnz,
                                              M.indptr.astype(np.int64) + 1,
                                              M.indices.astype(np.int32) + 1, M.data)
    if not ok:
        return None, False
    F = sp.csr_matrix((coef, ja.astype(np.int64) - 1, iat - 1), shape=(n, n))
    return F, True


def read_matrix_bin(path):
    """example_cpp binary CSR (Cpp_EMIN/readMat.cpp) -> scipy CSR."""
    h = C.c_void_p()
    check(load().chronos_read_matrix_bin(os.fsencode(path), C.byref(h)))
    return _CsrHandle.take(h)


def read_ext_bin(path):
    """Chronos .Ext_bin matrix (DumpChronos.cpp) -> scipy CSR."""
    h = C.c_void_p()
    check(load().chronos_read_ext_bin(os.fsencode(path), C.byref(h)))
    return _CsrHandle.take(h)


def write_ext_bin(path, A):
    n, iat, ja, val = _csr(A, A.shape[1])
    check(load().chronos_write_ext_bin(os.fsencode(path), n, A.shape[1], _pi(iat), _pi(ja),
                                       _pd(val)))


def read_tv_ext_bin(path):
    """Chronos .Ext_bin test space -> n x ntv array (ntv = 0 for a header-only file)."""
    n, ntv = C.c_int(), C.c_int()
    check(load().chronos_read_tv_ext_bin(os.fsencode(path), C.byref(n), C.byref(ntv), None))
    TV = np.zeros(max(n.value * ntv.value, 1))
    check(load().chronos_read_tv_ext_bin(os.fsencode(path), C.byref(n), C.byref(ntv), _pd(TV)))
    return TV[:n.value * ntv.value].reshape(ntv.value, n.value).T.copy()


def write_tv_ext_bin(path, TV):
    TV = np.asarray(TV, dtype=np.float64)
    if TV.ndim == 1:
        TV = TV[:, None]
    col = np.ascontiguousarray(TV.T).ravel()
    check(load().chronos_write_tv_ext_bin(os.fsencode(path), TV.shape[0], TV.shape[1], _pd(col)))


def fsai_pattern(A, nstep=15, step_size=1, eps=1e-3, nthread=1, fsai_fabs=0):
    """Host adaptive pattern search (no GPU): (G with host FP64 values, posdef)."""
    n, ip, ix, dv = _csr(A)
    ok = C.c_int()
    h = C.c_void_p()
    check(load().chronos_fsai_pattern(n, _pi(ip), _pi(ix), _pd(dv), nstep, step_size, eps,
                                      nthread, fsai_fabs, C.byref(ok), C.byref(h)))
    return _CsrHandle.take(h), bool(ok.value)


def fsai_numeric(A, G, base=1, precision=CHRONOS_FP64, stream=None):
    """GPU numeric phase on the pattern of G (rows: strictly-lower ascending,
    diagonal last), passed to chronos_fsai_numeric as 1-based (the MEX
    layout, base=1) or 0-based (base=0) CSR.  Returns (values in G's order
    as float64, or float32 for precision=CHRONOS_FP32; is_posdef).  stream:
    a cudaStream_t handle as an int (e.g. torch's stream.cuda_stream) or None."""
    A = sp.csr_matrix(A)
    A.sort_indices()
    G = sp.csr_matrix(G)
    n = A.shape[0]
    out = np.zeros(G.nnz, np.float64 if precision == CHRONOS_FP64 else np.float32)
    ok = C.c_int()
    iatA = A.indptr.astype(np.int64) + base
    jaA = A.indices.astype(np.int32) + base
    iatG = G.indptr.astype(np.int64) + base
    jaG = G.indices.astype(np.int32) + base
    dA = np.ascontiguousarray(A.data, np.float64)
    check(load().chronos_fsai_numeric(n, base, _pi64(iatA), _pi(jaA), _pd(dA), _pi64(iatG),
                                      _pi(jaG), precision, out.ctypes.data_as(C.c_void_p),
                                      C.byref(ok), _stream(stream)))
    return out, bool(ok.value)


def fsai_numeric_batch(As, Gs, tile_set=-1):
    """GPU FSAI numeric phase of several problems in one batched launch per
    tile size (chronos_fsai_numeric_batch).  Returns (list of value arrays in
    each G's order, list of is_posdef, the tile set run)."""
    mats = [_csr(A) for A in As]
    Gs = [sp.csr_matrix(G) for G in Gs]
    npb = len(mats)
    P = C.c_void_p * npb
    gp = [np.ascontiguousarray(G.indptr, dtype=np.int32) for G in Gs]
    gi = [np.ascontiguousarray(G.indices, dtype=np.int32) for G in Gs]
    outs = [np.zeros(max(G.nnz, 1)) for G in Gs]
    ok = np.zeros(npb, np.int32)
    used = C.c_int(-1)
    n = np.array([m[0] for m in mats], dtype=np.int32)
    check(load().chronos_fsai_numeric_batch(
        npb, _pi(n), P(*[m[1].ctypes.data for m in mats]), P(*[m[2].ctypes.data for m in mats]),
        P(*[m[3].ctypes.data for m in mats]), P(*[a.ctypes.data for a in gp]),
        P(*[a.ctypes.data for a in gi]), P(*[o.ctypes.data for o in outs]), _pi(ok), tile_set,
        C.byref(used)))
    return [o[:G.nnz] for o, G in zip(outs, Gs)], [bool(v) for v in ok], used.value


def _stream(s):
    """cudaStream_t argument from None (the legacy default stream), an int
    handle or an object with a cuda_stream attribute (torch.cuda.Stream)."""
    if s is None:
        return None
    return C.c_void_p(int(getattr(s, "cuda_stream", s)))


# ---------------------------------------------------------------------------
# Coarsening, prolongation, Galerkin, coarse factor
# ---------------------------------------------------------------------------

def coarsen(A, prm=None, rng_skip=0):
    """SoC + PMIS on the host: (fcnode numbered as the reference, nc, S)."""
    prm = prm or params()
    n, ip, ix, dv = _csr(A)
    fc = np.zeros(n, np.int32)
    nc = C.c_int()
    h = C.c_void_p()
    check(load().chronos_coarsen(C.byref(prm), n, _pi(ip), _pi(ix), _pd(dv), rng_skip, _pi(fc),
                                 C.byref(nc), C.byref(h)))
    return fc.astype(np.int64), nc.value, _CsrHandle.take(h)


def device_bytes():
    """Device memory held by the library in this process (chronos_device_bytes)."""
    v = C.c_int64()
    check(load().chronos_device_bytes(C.byref(v)))
    return v.value


def coarsen_device(A, prm=None, rng_skip=0):
    """DOM strength + PMIS on the GPU: (fcnode, nc, S pattern), the same
    splitting as coarsen()."""
    prm = prm or params()
    n, ip, ix, dv = _csr(A)
    fc = np.zeros(n, np.int32)
    nc = C.c_int()
    h = C.c_void_p()
    check(load().chronos_coarsen_device(C.byref(prm), n, _pi(ip), _pi(ix), _pd(dv), rng_skip,
                                        _pi(fc), C.byref(nc), C.byref(h)))
    return fc.astype(np.int64), nc.value, _CsrHandle.take(h)


def bamg(S, fcnode, TV, prm=None, device=False, max_neigh=0):
    """BAMG prolongation: (P, c_mark) from the host restatement, or with
    device=True from the GPU (chronos_bamg_device; the same bits; max_neigh
    caps a GPU thread's neighbourhood, 0 automatic), then (P, c_mark, rows
    computed on the host)."""
    prm = prm or params()
    S = sp.csr_matrix(S)
    S.sort_indices()
    n = S.shape[0]
    ip = S.indptr.astype(np.int32)
    ix = S.indices.astype(np.int32)
    fc = np.ascontiguousarray(fcnode, dtype=np.int32)
    TV = np.asfortranarray(np.asarray(TV, dtype=np.float64).reshape(n, -1))
    ntv = TV.shape[1]
    tvc = np.ascontiguousarray(TV.T).ravel()      # column-major
    cm = np.zeros(n, np.int32)
    h = C.c_void_p()
    if device:
        hr = C.c_int(-1)
        check(load().chronos_bamg_device(C.byref(prm), n, _pi(ip), _pi(ix), _pi(fc), ntv, _pd(tvc),
                                         _pi(cm), max_neigh, C.byref(h), C.byref(hr)))
        return _CsrHandle.take(h), cm, hr.value
    check(load().chronos_bamg(C.byref(prm), n, _pi(ip), _pi(ix), _pi(fc), ntv, _pd(tvc), _pi(cm),
                              C.byref(h)))
    return _CsrHandle.take(h), cm


def emin_pattern(S, P, fcnode, kpow=2, nnzr_max=30, nnzr_min=None):
    """EMIN prolongation pattern on the GPU (chronos_emin_pattern; replaces
    MEX_cptProlPatt as prolong.m:222 calls it).  S: strength matrix with
    values, P: n x nc prolongation, fcnode as coarsen returns it; nnzr_min
    defaults to ntv as prolong.m passes it (give it explicitly).  Returns
    (pattern n x nc with the MEX's values, rows computed on the host)."""
    S = sp.csr_matrix(S)
    S.sort_indices()
    P = sp.csr_matrix(P)
    P.sort_indices()
    n, nc = P.shape
    if S.shape != (n, n) or np.size(fcnode) != n:
        raise ValueError("S must be n x n and fcnode of length n")
    if nnzr_min is None:
        raise ValueError("nnzr_min (the number of test vectors) is required")
    fc = np.ascontiguousarray(fcnode, dtype=np.int32)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
    si, sx, sv = i32(S.indptr), i32(S.indices), np.ascontiguousarray(S.data, np.float64)
    pi, px, pv = i32(P.indptr), i32(P.indices), np.ascontiguousarray(P.data, np.float64)
    h = C.c_void_p()
    hr = C.c_int(0)
    check(load().chronos_emin_pattern(kpow, n, nc, _pi(si), _pi(sx), _pd(sv), _pi(pi), _pi(px),
                                      _pd(pv), _pi(fc), nnzr_max, nnzr_min, C.byref(h),
                                      C.byref(hr)))
    return _CsrHandle.take(h), hr.value


def emin(A, P, pattern, fcnode, TV, prm=None, spd=True):
    """Energy minimisation of P on the pattern on the GPU (chronos_emin;
    replaces EMIN_Prolong_compute / EMIN_ImpProl, matrix-free path, Jacobi,
    SPD).  Returns (P n x nc, info[12]): info[7] CG iterations, info[6] rows
    whose constraint block took the SVD branch."""
    prm = prm or params()
    n, ip, ix, dv = _csr(A)
    P = sp.csr_matrix(P)
    P.sort_indices()
    nc = P.shape[1]
    T = sp.csr_matrix(pattern)
    T.sort_indices()
    if P.shape[0] != n or T.shape != P.shape or np.size(fcnode) != n:
        raise ValueError("P and the pattern must be n x nc, fcnode of length n")
    TV = np.asarray(TV, dtype=np.float64).reshape(n, -1)
    ntv = TV.shape[1]
    tvc = np.ascontiguousarray(TV.T).ravel()           # column-major
    fc = np.ascontiguousarray(fcnode, dtype=np.int32)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
    pi, px, pv = i32(P.indptr), i32(P.indices), np.ascontiguousarray(P.data, np.float64)
    ti, tx = i32(T.indptr), i32(T.indices)
    info = np.zeros(12)
    h = C.c_void_p()
    check(load().chronos_emin(C.byref(prm), n, _pi(ip), _pi(ix), _pd(dv), nc, _pi(pi), _pi(px),
                              _pd(pv), _pi(ti), _pi(tx), _pi(fc), ntv, _pd(tvc),
                              1 if spd else 0, C.byref(h), _pd(info)))
    return _CsrHandle.take(h), info


def galerkin(A, P):
    """GPU Galerkin product P'*(A*P) (exact zeros dropped, sorted rows)."""
    n, ip, ix, dv = _csr(A)
    P = sp.csr_matrix(P)
    nc = P.shape[1]
    pp = P.indptr.astype(np.int32)
    px = P.indices.astype(np.int32)
    pv = np.ascontiguousarray(P.data, np.float64)
    nnz = C.c_int64()
    plan = C.c_void_p()
    lib = load()
    check(lib.chronos_galerkin_compute(n, nc, _pi(ip), _pi(ix), _pd(dv), _pi(pp), _pi(px),
                                       _pd(pv), C.byref(nnz), C.byref(plan)))
    try:
        iat = np.zeros(nc + 1, np.int32)
        ja = np.zeros(max(nnz.value, 1), np.int32)
        v = np.zeros(max(nnz.value, 1), np.float64)
        check(lib.chronos_galerkin_fetch(plan, _pi(iat), _pi(ja), _pd(v)))
    finally:
        lib.chronos_galerkin_free(plan)
    return sp.csr_matrix((v[:nnz.value], ja[:nnz.value], iat), shape=(nc, nc))


def dense_chol(A):
    """GPU dense FP64 Cholesky: lower L with A = L L'."""
    A = np.asfortranarray(np.asarray(A, dtype=np.float64))
    n = A.shape[0]
    a = np.ascontiguousarray(A.T).ravel()     # column-major
    L = np.zeros(n * n, np.float64)
    check(load().chronos_dense_chol(n, _pd(a), _pd(L)))
    return L.reshape(n, n).T.copy()


def spmv(A, x, precision=CHRONOS_FP64, format=0, lanes=0):
    """y = A x on the GPU through the V-cycle's apply kernels (format: 0 tuned,
    1 row-grouped CSR, 2 sliced ELL; lanes > 0 forces the CSR lanes per row)."""
    n, ip, ix, dv = _csr(A)
    x = np.ascontiguousarray(x, np.float64)
    y = np.zeros(n, np.float64)
    check(load().chronos_spmv(n, A.shape[1], _pi(ip), _pi(ix), _pd(dv), _pd(x), _pd(y), precision,
                              format, lanes))
    return y


def diag_fix(A):
    """computeAMG.m:5-10 on the GPU: diagonal entries equal to 1 become
    lambda_max(A)/10.  Returns a new matrix."""
    A = sp.csr_matrix(A, copy=True)
    A.sort_indices()
    n, ip, ix, dv = _csr(A)
    dv = dv.copy()
    check(load().chronos_diag_fix(n, _pi(ip), _pi(ix), _pd(dv)))
    return sp.csr_matrix((dv, ix, ip), shape=A.shape)


# ---------------------------------------------------------------------------
# Hierarchy, V-cycle, Krylov
# ---------------------------------------------------------------------------

class Hierarchy:
    """Handle of a GPU AMG hierarchy (chronos_hier)."""

    def __init__(self, A, TV0=None, prm=None):
        self._lib = load()
        self.prm = prm or params()
        n, ip, ix, dv = _csr(A)
        self.n = n
        if TV0 is None:
            ntv0, tv = 0, np.zeros(1)
        else:
            TV0 = np.asarray(TV0, dtype=np.float64).reshape(n, -1)
            ntv0 = TV0.shape[1]
            tv = np.ascontiguousarray(TV0.T).ravel()
        h = C.c_void_p()
        check(self._lib.chronos_amg_setup(C.byref(self.prm), n, _pi(ip), _pi(ix), _pd(dv), ntv0,
                                          _pd(tv), C.byref(h)))
        self._h = h

    @classmethod
    def with_prolongation(cls, A, prolong, prm=None):
        """cpt_aspAMG with every level's P from the caller (chronos_amg_setup_prolong):
        `prolong` is a callable (level, A_level) -> P (scipy CSR, n x nc), called
        for each level that is not the coarsest with the 1-based level number and
        the level's operator, or a list of P matrices taken in order.  The
        library computes FSAI, omega, the Galerkin products and the coarse
        factor; coarsening and the prolongation stay with the caller, as
        cpt_aspAMG.m:224-225 calls prolong(...) on the host."""
        from ._lib import PROLONG_FN
        self = cls.__new__(cls)
        self._lib = load()
        self.prm = prm or params()
        n, ip, ix, dv = _csr(A)
        self.n = n
        if not callable(prolong):
            plist = list(prolong)
            prolong = lambda level, Al: plist[level - 1]   # noqa: E731
        keep = []          # the arrays of the latest P stay alive until the next call
        errors = []

        def cb(ctx, level, nl, iat, ja, val, out):
            try:
                nnz = iat[nl]
                rp = np.ctypeslib.as_array(iat, shape=(nl + 1,)).copy()
                Al = sp.csr_matrix((np.ctypeslib.as_array(val, shape=(max(nnz, 1),))[:nnz].copy(),
                                    np.ctypeslib.as_array(ja, shape=(max(nnz, 1),))[:nnz].copy(),
                                    rp), shape=(nl, nl))
                P = sp.csr_matrix(prolong(level, Al))
                if P.shape[0] != nl:
                    # the library reads n + 1 row pointers from the returned array
                    raise ChronosError(-1, f"prolongation of level {level} has {P.shape[0]} "
                                           f"rows, the level has {nl}")
                P.sort_indices()
                pp = np.ascontiguousarray(P.indptr, dtype=np.int32)
                pi = np.ascontiguousarray(P.indices, dtype=np.int32)
                pv = np.ascontiguousarray(P.data, dtype=np.float64)
                if pi.size == 0:
                    pi, pv = np.zeros(1, np.int32), np.zeros(1)
                keep[:] = [pp, pi, pv]
                out[0].nc = int(P.shape[1])
                out[0].iat_P_h = _pi(pp)
                out[0].ja_P_h = _pi(pi)
                out[0].val_P_h = _pd(pv)
                return 0
            except Exception as e:       # noqa: BLE001 -- reported after the call
                errors.append(e)
                return -1

        fn = PROLONG_FN(cb)
        h = C.c_void_p()
        code = self._lib.chronos_amg_setup_prolong(C.byref(self.prm), n, _pi(ip), _pi(ix), _pd(dv),
                                                   fn, None, C.byref(h))
        if errors:
            raise errors[0]
        check(code)
        self._h = h
        return self

    def save(self, path):
        """Writes the hierarchy to a file that Hierarchy.load reads back
        without the setup (chronos_hier_save)."""
        check(self._lib.chronos_hier_save(self._h, os.fsencode(path)))

    @classmethod
    def load(cls, path):
        """A hierarchy rebuilt from a file written by save (chronos_hier_load)."""
        self = cls.__new__(cls)
        self._lib = load()
        h = C.c_void_p()
        check(self._lib.chronos_hier_load(os.fsencode(path), C.byref(h)))
        self._h = h
        info = chronos_level_info()
        check(self._lib.chronos_hier_level_info(h, 0, C.byref(info)))
        self.n = info.n
        self.prm = None
        return self

    def close(self):
        if getattr(self, "_h", None):
            self._lib.chronos_hier_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def nlevels(self):
        v = C.c_int()
        check(self._lib.chronos_hier_nlevels(self._h, C.byref(v)))
        return v.value

    def level_info(self, level):
        info = chronos_level_info()
        check(self._lib.chronos_hier_level_info(self._h, level, C.byref(info)))
        return {"n": info.n, "nnz_A": info.nnz_A, "nnz_G": info.nnz_G, "nnz_P": info.nnz_P,
                "nc": info.nc, "omega": info.omega, "lambda": info.lambda_,
                "threads_per_row": info.threads_per_row, "block_rows": info.block_rows,
                "sell_mask": info.sell_mask}

    def amg_info(self):
        """Hierarchy statistics as get_AMG_info.m:1-81 gathers them: per level
        the rows nn, entries nt, coarse size nc and prolongation entries nt_P
        (smoothing levels) or the dense factor's entries nt_L (coarsest), and
        on the first level the grid and operator complexities sum(nn)/nn_1
        and sum(nt)/nt_1."""
        out = []
        for l in range(self.nlevels):
            i = self.level_info(l)
            d = {"nn": i["n"], "nt": i["nnz_A"], "omega": i["omega"]}
            if l < self.nlevels - 1:
                d.update(nc=i["nc"], nt_P=i["nnz_P"], nt_G=i["nnz_G"])
            else:
                d.update(nt_L=i["n"] * (i["n"] + 1) // 2)
            out.append(d)
        out[0]["grid_comp"] = sum(d["nn"] for d in out) / out[0]["nn"]
        out[0]["oper_comp"] = sum(d["nt"] for d in out) / out[0]["nt"]
        return out

    def export(self, level, which):
        nr, ncl, nnz = C.c_int(), C.c_int(), C.c_int64()
        w = C.c_char(which.encode() if isinstance(which, str) else which)
        check(self._lib.chronos_hier_export(self._h, level, w, C.byref(nr), C.byref(ncl),
                                            C.byref(nnz), None, None, None))
        iat = np.zeros(nr.value + 1, np.int32)
        ja = np.zeros(max(nnz.value, 1), np.int32)
        v = np.zeros(max(nnz.value, 1), np.float64)
        check(self._lib.chronos_hier_export(self._h, level, w, C.byref(nr), C.byref(ncl),
                                            C.byref(nnz), _pi(iat), _pi(ja), _pd(v)))
        return sp.csr_matrix((v[:nnz.value], ja[:nnz.value], iat), shape=(nr.value, ncl.value))

    def dump_ext_bin(self, level, which, path):
        """Writes operator `which` ('A', 'G', 'P') of a level in .Ext_bin."""
        w = C.c_char(which.encode() if isinstance(which, str) else which)
        check(self._lib.chronos_hier_dump_ext_bin(self._h, level, w, os.fsencode(path)))

    def setup_times(self):
        """Setup phases in seconds; the phases other than "total" sum to it."""
        keys = ["fsai_pattern", "fsai_numeric", "omega", "coarsen", "prolong", "galerkin",
                "coarse_factor", "total", "uploads", "layouts", "autotune", "other"]
        t = np.zeros(len(keys))
        check(self._lib.chronos_hier_setup_phases(self._h, _pd(t), len(keys)))
        return dict(zip(keys, t.tolist()))

    def profile(self, reps=20):
        """CUDA-event timings (ms) and algorithmic bytes of the hot kernels."""
        from ._lib import chronos_profile
        p = chronos_profile()
        check(self._lib.chronos_hier_profile(self._h, reps, C.byref(p)))
        return {k: getattr(p, k) for k, _ in chronos_profile._fields_}

    def _operator(self, A):
        """0-based CSR pointers of an operator of the hierarchy's level-1 size.
        The C ABI reads n + 1 row pointers from the caller's array, so the
        size is checked here, before the call."""
        if A.shape != (self.n, self.n):
            raise ChronosError(-1, f"operator of shape {A.shape}, the hierarchy has n = {self.n}")
        _, ip, ix, dv = _csr(A)
        self._op_keep = (ip, ix, dv)
        return (_pi(ip), _pi(ix), _pd(dv))

    def vcycle(self, b, stream=None):
        b = np.asarray(b, dtype=np.float64)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        bc = np.ascontiguousarray(b.T if b.ndim == 2 else b).ravel()
        x = np.zeros_like(bc)
        check(self._lib.chronos_vcycle(self._h, _pd(bc), _pd(x), nrhs, _stream(stream)))
        return x if b.ndim == 1 else x.reshape(nrhs, self.n).T

    def vcycle_dev(self, b_ptr, x_ptr, precision=CHRONOS_FP64, nrhs=1, stream=None):
        """AMG_Vcycle on device vectors (chronos_vcycle_dev): b_ptr, x_ptr are
        device addresses of n x nrhs column-major double (CHRONOS_FP64) or
        float (CHRONOS_FP32) arrays; ordered on stream."""
        check(self._lib.chronos_vcycle_dev(self._h, precision, C.c_void_p(b_ptr),
                                           C.c_void_p(x_ptr), nrhs, _stream(stream)))

    def pcg(self, b, x0=None, itmax=1000, tol=1e-8, A=None, stream=None):
        """PCG_CJ; A (optional) is the operator prodA (0-based CSR of the
        level-1 size), else the hierarchy's level-1 operator."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        it, flag, sec = C.c_int(), C.c_int(), C.c_double()
        rv = np.zeros(max(itmax, 0) + 1)
        if A is not None:
            ops = self._operator(A)
        else:
            ops = (None, None, None)
        check(self._lib.chronos_pcg(self._h, *ops, _pd(b), _pd(x), itmax, tol, C.byref(it),
                                    _pd(rv), C.byref(flag), C.byref(sec), _stream(stream)))
        return x, it.value, rv[:it.value + 1], flag.value, sec.value

    def pcg_host(self, b, x, itmax=1000, tol=1e-8):
        """PCG on caller-owned host vectors, in place: b and x (x0 on entry,
        the solution on return) are C-contiguous float64 arrays of length n,
        passed to chronos_pcg without a copy, so pinned (page-locked) buffers
        stay pinned for the library's host-device copies."""
        for v in (b, x):
            if not (isinstance(v, np.ndarray) and v.dtype == np.float64 and v.ndim == 1
                    and v.flags.c_contiguous and v.size == self.n):
                raise ChronosError(-1, "pcg_host: b and x must be contiguous "
                                   "float64 arrays of length n")
        it, flag, sec = C.c_int(), C.c_int(), C.c_double()
        check(self._lib.chronos_pcg(self._h, None, None, None, _pd(b), _pd(x), itmax, tol,
                                    C.byref(it), None, C.byref(flag), C.byref(sec), None))
        return it.value, flag.value, sec.value

    def pcg_dev(self, b_ptr, x_ptr, itmax=1000, tol=1e-8, stream=None):
        """PCG on device FP64 vectors (raw pointers, e.g. torch tensor.data_ptr()),
        ordered on `stream` (torch.cuda.Stream, an int handle, or None)."""
        it, flag, sec = C.c_int(), C.c_int(), C.c_double()
        check(self._lib.chronos_pcg_dev(self._h, C.c_void_p(b_ptr), C.c_void_p(x_ptr), itmax, tol,
                                        C.byref(it), None, C.byref(flag), C.byref(sec),
                                        _stream(stream)))
        return it.value, flag.value, sec.value

    def pcg_block(self, B, X0=None, itmax=1000, tol=1e-8, stream=None):
        B = np.asarray(B, dtype=np.float64)
        nrhs = B.shape[1]
        bc = np.ascontiguousarray(B.T).ravel()
        xc = np.zeros_like(bc) if X0 is None else np.ascontiguousarray(np.asarray(X0).T).ravel()
        its = np.zeros(nrhs, np.int32)
        fl = np.zeros(nrhs, np.int32)
        sec = C.c_double()
        check(self._lib.chronos_pcg_block(self._h, nrhs, _pd(bc), _pd(xc), itmax, tol, _pi(its),
                                          _pi(fl), C.byref(sec), _stream(stream)))
        return xc.reshape(nrhs, self.n).T, its, fl, sec.value

    def sqmr(self, b, tol=1e-6, itmax=100, x0=None, A=None):
        """SQMR with the V-cycle as left preconditioner; A (optional) is the
        operator, else the level-1 operator of the hierarchy."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        it, info, rel = C.c_int(), C.c_int(), C.c_double()
        if A is not None:
            ops = self._operator(A)
        else:
            ops = (None, None, None)
        check(self._lib.chronos_sqmr(self._h, *ops, _pd(b), _pd(x), itmax, tol, C.byref(it),
                                     C.byref(rel), C.byref(info)))
        return x, info.value, rel.value, it.value

    def gmres(self, b, restart=50, tol=1e-6, maxit=2, x0=None, A=None):
        """gmres_RIGHT with the V-cycle as right preconditioner; A (optional)
        is the operator, else the level-1 operator of the hierarchy.  Returns
        (x, flag, relres, (outer, inner), resvec)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        if A is not None:
            ops = self._operator(A)
        else:
            ops = (None, None, None)
        io, ii, fl, nrv = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        rel = C.c_double()
        rv = np.zeros(max(restart, 0) * max(maxit, 0) + 1)
        check(self._lib.chronos_gmres(self._h, *ops, _pd(b), _pd(x), restart, tol, maxit,
                                      C.byref(io), C.byref(ii), C.byref(rel), C.byref(fl),
                                      _pd(rv), C.byref(nrv)))
        return x, fl.value, rel.value, (io.value, ii.value), rv[:nrv.value]

    def adjoint_grad(self, u, g, itmax=1000, tol=1e-10):
        """dJ/dA on A's pattern for J with dJ/du = g (A SPD): returns
        (lambda, grad values in A's CSR order, iterations)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        g = np.ascontiguousarray(g, dtype=np.float64)
        lam = np.zeros(self.n)
        A0 = self.level_info(0)
        grad = np.zeros(max(A0["nnz_A"], 1))
        it = C.c_int()
        check(self._lib.chronos_adjoint_grad(self._h, _pd(u), _pd(g), itmax, tol, _pd(lam),
                                             _pd(grad), C.byref(it)))
        return lam, grad[:A0["nnz_A"]], it.value


class Batch:
    """Independent problems of uneven sizes (chronos_batch): one hierarchy per
    problem; by default (batch_grouped = 1) one launch sequence serves the
    whole batch (stacked level operators, per-problem PCG_CJ scalars), else
    one conditional-graph launch per problem on its own stream."""

    def __init__(self, As, prm=None):
        self._lib = load()
        self.prm = prm or params(ntv=1)
        mats = [_csr(A) for A in As]
        self.ns = [m[0] for m in mats]
        self._keep = mats
        npb = len(mats)
        n = np.array(self.ns, dtype=np.int32)
        P = C.c_void_p * npb
        iat = P(*[m[1].ctypes.data for m in mats])
        ja = P(*[m[2].ctypes.data for m in mats])
        val = P(*[m[3].ctypes.data for m in mats])
        h = C.c_void_p()
        check(self._lib.chronos_batch_setup(C.byref(self.prm), npb, _pi(n), iat, ja, val,
                                            C.byref(h)))
        self._h = h
        self._keep = None

    def close(self):
        if getattr(self, "_h", None):
            self._lib.chronos_batch_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def nlevels(self, p):
        nl, n0 = C.c_int(), C.c_int()
        check(self._lib.chronos_batch_info(self._h, p, C.byref(nl), C.byref(n0)))
        return nl.value

    def setup_times(self):
        """Hierarchy.setup_times' phases summed over the problems (thread time)."""
        keys = ["fsai_pattern", "fsai_numeric", "omega", "coarsen", "prolong", "galerkin",
                "coarse_factor", "total", "uploads", "layouts", "autotune", "other"]
        t = np.zeros(len(keys))
        check(self._lib.chronos_batch_setup_phases(self._h, _pd(t), len(keys)))
        return dict(zip(keys, t.tolist()))

    def setup_wall(self):
        """The batch setup's wall clock (s) by stage."""
        keys = ["first_levels", "fsai_numeric_batched", "rest", "tune_group", "total"]
        t = np.zeros(len(keys))
        check(self._lib.chronos_batch_setup_wall(self._h, _pd(t)))
        return dict(zip(keys, t.tolist()))

    def solve(self, bs, itmax=1000, tol=1e-8):
        """Returns (xs, iters, flags, seconds)."""
        npb = len(self.ns)
        bs = [np.ascontiguousarray(b, dtype=np.float64) for b in bs]
        xs = [np.zeros(n) for n in self.ns]
        P = C.c_void_p * npb
        its = np.zeros(npb, np.int32)
        fl = np.zeros(npb, np.int32)
        sec = C.c_double()
        check(self._lib.chronos_batch_solve(self._h, P(*[b.ctypes.data for b in bs]),
                                            P(*[x.ctypes.data for x in xs]), itmax, tol, _pi(its),
                                            _pi(fl), C.byref(sec)))
        return xs, its, fl, sec.value


def cpt_aspAMG(param, A, TV0=None):
    """cpt_aspAMG.m:1: builds the hierarchy (param: chronos_params)."""
    return Hierarchy(A, TV0, param)


def AMG_Vcycle(hrc, b):
    """AMG_Vcycle.m (x0 absent): x = M^{-1} b."""
    return hrc.vcycle(b)


def PCG_CJ(hrc, b, x0=None, itmax=15000, tol=1e-8):
    """PCG_CJ.m:1: returns (x, iter, resvec, flag)."""
    x, it, rv, flag, _ = hrc.pcg(b, x0, itmax, tol)
    return x, it, rv, flag


def SQMR(hrc, rhs, tol=1e-6, itmax=100, x0=None, A=None):
    """SQMR.m:1 with the V-cycle as left preconditioner: (x, info, relres, niter)."""
    return hrc.sqmr(rhs, tol, itmax, x0, A)


def gmres_RIGHT(hrc, b, restart=None, tol=1e-6, maxit=None, x0=None, A=None):
    """gmres_RIGHT.m:7 with the V-cycle as the right preconditioner M:
    (x, flag, relres, iter, resvec), iter = (outer, inner).  restart None is
    the unrestarted method (restart = n); maxit None is
    min(ceil(n/restart), 10) cycles, or min(n, 10) iterations unrestarted, as
    gmres_RIGHT.m:98-157 chooses."""
    n = hrc.n
    if restart is None or restart == n:
        inner = min(n, 10) if maxit is None else min(int(maxit), n)
        return hrc.gmres(b, restart=inner, tol=tol, maxit=1, x0=x0, A=A)
    if maxit is None:
        maxit = min(-(-n // max(int(restart), 1)), 10)
    return hrc.gmres(b, restart=min(int(restart), n), tol=tol, maxit=int(maxit), x0=x0, A=A)
