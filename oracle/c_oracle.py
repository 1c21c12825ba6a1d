"""ctypes wrapper of oracle/_build/liboracle.so (chronos_oracle.c) and the FP64
reference pipeline used for the CPU baseline.

ORACLE TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and the CPU
baseline / reference arm of bench.py use this module.

reference_hierarchy() builds the FP64 hierarchy the way the reference does,
with the reference's own C++ kernels where it has them (compute_local_fsai,
BAMG from oracle/_ref) and the restatements of its MATLAB glue elsewhere
(strength of connection in numpy, PMIS in C, Galerkin by scipy's Gustavson
product, eigs by ARPACK, chol by LAPACK).  pcg() then runs PCG_CJ with the
V-cycle in C with OpenMP.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import scipy.sparse as sp

from . import amg_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")


class _ocsr(C.Structure):
    _fields_ = [("nrows", C.c_int), ("ncols", C.c_int), ("rp", C.POINTER(C.c_int64)),
                ("ci", C.POINTER(C.c_int)), ("v", C.POINTER(C.c_double))]


class _olevel(C.Structure):
    _fields_ = [("n", C.c_int), ("A", _ocsr), ("G", _ocsr), ("Gt", _ocsr), ("P", _ocsr),
                ("Pt", _ocsr), ("omega", C.c_double), ("L", C.POINTER(C.c_double)),
                ("nupre", C.c_int), ("nupost", C.c_int)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        lib.oracle_set_threads.argtypes = [C.c_int]
        lib.oracle_spmv.argtypes = [C.POINTER(_ocsr), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        lib.oracle_vcycle.argtypes = [C.c_int, C.POINTER(_olevel), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double)]
        lib.oracle_pcg_cj.argtypes = [C.c_int, C.POINTER(_olevel), C.POINTER(_ocsr),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int,
                                      C.c_double, C.POINTER(C.c_int), C.POINTER(C.c_double)]
        lib.oracle_pcg_cj.restype = C.c_int
        lib.oracle_pmis.argtypes = [C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_int),
                                    C.POINTER(C.c_double), C.POINTER(C.c_int)]
        lib.oracle_pmis.restype = C.c_int
        _lib = lib
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class _Keep:
    """Holds the numpy arrays the C structs point into."""

    def __init__(self):
        self.arrays = []

    def csr(self, M):
        M = sp.csr_matrix(M)
        rp = np.ascontiguousarray(M.indptr, dtype=np.int64)
        ci = np.ascontiguousarray(M.indices, dtype=np.int32)
        v = np.ascontiguousarray(M.data, dtype=np.float64)
        self.arrays += [rp, ci, v]
        return _ocsr(M.shape[0], M.shape[1], rp.ctypes.data_as(C.POINTER(C.c_int64)),
                     ci.ctypes.data_as(C.POINTER(C.c_int)), _dp(v))


class CHierarchy:
    """An oracle hierarchy (amg_oracle.Hierarchy) mirrored into C structs."""

    def __init__(self, H, threads=0):
        self.lib = load()
        self.lib.oracle_set_threads(int(threads))
        self.keep = _Keep()
        lv = (_olevel * len(H.levels))()
        for k, L in enumerate(H.levels):
            lv[k].n = L.A.shape[0]
            lv[k].A = self.keep.csr(L.A)
            lv[k].nupre, lv[k].nupost = L.nupre, L.nupost
            if L.L is not None:
                Lc = np.asfortranarray(L.L).ravel(order="F")
                self.keep.arrays.append(Lc)
                lv[k].L = _dp(Lc)
            else:
                lv[k].G = self.keep.csr(L.G)
                lv[k].Gt = self.keep.csr(L.G.T.tocsr())
                lv[k].P = self.keep.csr(L.P)
                lv[k].Pt = self.keep.csr(L.P.T.tocsr())
                lv[k].omega = L.omega
        self.levels = lv
        self.nlev = len(H.levels)
        self.A = self.keep.csr(H.levels[0].A)
        self.n = H.levels[0].A.shape[0]

    def vcycle(self, b):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b)
        self.lib.oracle_vcycle(self.nlev, self.levels, _dp(b), _dp(x))
        return x

    def pcg(self, b, x0=None, itmax=1000, tol=1e-8):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros(self.n) if x0 is None else np.array(x0, dtype=np.float64)
        rv = np.zeros(itmax + 1)
        it = C.c_int()
        flag = self.lib.oracle_pcg_cj(self.nlev, self.levels, C.byref(self.A), _dp(b), _dp(x),
                                      itmax, tol, C.byref(it), _dp(rv))
        return x, it.value, rv[:it.value + 1], flag


def pmis_c(S, fcnode, rnd):
    S = sp.csr_matrix(S)
    rp = np.ascontiguousarray(S.indptr, dtype=np.int64)
    ci = np.ascontiguousarray(S.indices, dtype=np.int32)
    fc = np.ascontiguousarray(fcnode, dtype=np.int32).copy()
    r = np.ascontiguousarray(rnd, dtype=np.float64)
    nc = load().oracle_pmis(S.shape[0], rp.ctypes.data_as(C.POINTER(C.c_int64)),
                            ci.ctypes.data_as(C.POINTER(C.c_int)), _dp(r),
                            fc.ctypes.data_as(C.POINTER(C.c_int)))
    return fc.astype(np.int64), nc


def reference_hierarchy(A, TV0, prm, on_level=None):
    """cpt_aspAMG restated with the reference's own FSAI/BAMG C++ and the C
    PMIS (same algorithm as amg_oracle.cpt_pmis, faster)."""
    rng = O.MatlabRand()
    A = sp.csr_matrix(A)
    A.sort_indices()
    n = A.shape[0]
    ntv = prm["tspace"]["ntv"]
    TV0 = np.zeros((n, 0)) if TV0 is None else np.asarray(TV0, dtype=np.float64).reshape(n, -1)
    TV = np.zeros((n, ntv))
    nc0 = min(TV0.shape[1], ntv)
    TV[:, :nc0] = TV0[:, :nc0]
    if ntv > TV0.shape[1]:
        TV[:, TV0.shape[1]:] = rng.rand(n, ntv - TV0.shape[1]).reshape(n, -1)
    TV = O.qr_thin(TV)
    H = O.Hierarchy()
    level = 0
    while True:
        level += 1
        n = A.shape[0]
        if n <= prm["amg"]["maxCoarseSZ"] or level >= prm["amg"]["nLevMax"]:
            H.levels.append(O.Level(A=A, L=np.linalg.cholesky(A.toarray())))
            break
        G, omega, lam = O.smoother_afsai(A, prm["smoother"])
        TV = O.qr_thin(TV)
        fc0, _ = O.mark_isolated_nodes(A, np.zeros(n, dtype=np.int64))
        S = O.soc_dom(prm["coarsen"]["tau"], A) if prm["coarsen"]["SoC_type"].upper() == "DOM" \
            else O.soc_cla(prm["coarsen"]["tau"], A)
        fc, nc = pmis_c(S, fc0, rng.rand(n))
        P, _ = O.ref_bamg(prm["prolong"], nc, fc, S, TV)
        TV = TV[np.flatnonzero(fc > 0), :]
        Ac = O.galerkin(P, A)
        lev = O.Level(A=A, G=G, omega=omega, P=P, fcnode=fc, nupre=prm["smoother"]["nupre"],
                      nupost=prm["smoother"]["nupost"], lam=lam)
        H.levels.append(lev)
        if on_level:
            on_level(level, lev)
        A = Ac
    return H
