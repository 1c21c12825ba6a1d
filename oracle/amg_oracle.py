"""CPU oracle for ChronosLab's AMG-preconditioned SPD solve path.

ORACLE TEST INFRASTRUCTURE.  Only tests/, __graft_entry__.smoke() and the CPU
baseline / reference arm of bench.py import this module, and only as the
checker.  The chronoslab_b200 package never imports it.

FP64 restatement, in numpy/scipy, of the reference's MATLAB layer (which cannot
run here: no MATLAB/Octave), following the reference files line by line:

  PCG_CJ            sources/LinearSolver/PCG_CJ.m:1-73
  SQMR              sources/LinearSolver/SQMR.m:1-108
  AMG_Vcycle        sources/Preconditioner/AMG/aspAMG/AMG_Vcycle.m:1-54
  cpt_aspAMG        sources/Preconditioner/AMG/aspAMG/cpt_aspAMG.m:1-351
  smoother          sources/Preconditioner/AMG/smoother/smoother.m:33-87
  afsai_cpp         sources/Preconditioner/AMG/smoother/afsai_cpp.m:1-65
  coarsen           sources/Preconditioner/AMG/coarsen/coarsen.m:1-76
  mark_isolated     sources/Preconditioner/AMG/coarsen/mark_isolated_nodes.m:1-8
  cpt_SoC_dom/cla   sources/Preconditioner/AMG/coarsen/cpt_SoC_{dom,cla}.m
  cpt_PMIS          sources/Preconditioner/AMG/coarsen/cpt_PMIS.m:1-102
  cpt_ProlMEX_BAMG  sources/Preconditioner/AMG/prolong/cpt_ProlMEX_BAMG.m:1-72
  EMIN              sources/Preconditioner/AMG/prolong/prolong.m:207-235 with
                    EMIN/MEX_EMIN/MEX_cptProlPatt.cpp (pattern) and
                    EMIN/Cpp_EMIN/EMIN_matfree.cpp, DEFL_PCG_matfree.cpp,
                    gather_B_QR.cpp, KP_spmat.cpp, Orth_Q.cpp (energy minimisation)
  computeAMG        sources/utils/computeAMG.m:1-51
  mk_rbm_3d         sources/utils/mk_rbm_3d.m:1-27

The reference's own C++ kernels are used through oracle/_ref (built by
oracle/Makefile from the unmodified reference sources): compute_local_fsai
(FSAI), BAMG (prolongation), and the EMIN pattern and energy minimisation;
the EMIN restatement here (emin_pattern, emin_enhance) is checked against
the latter.  MATLAB built-ins are replaced by their
published counterparts: sparse products by scipy (Gustavson, exact zeros
dropped as MATLAB does), chol by numpy's LAPACK Cholesky, eigs by ARPACK
(scipy.sparse.linalg.eigsh), rand after rng(0) by MT19937 seeded 5489 with
53-bit doubles (numpy.random.RandomState(5489).random_sample), filled
column-major as MATLAB's rand(n,k).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np
import scipy.io
import scipy.linalg
import scipy.sparse as sp
import scipy.sparse.linalg as spla

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


# ----------------------------------------------------------------------------
# Parameter files (read_amg.m, read_smoother.m, read_tspace.m, read_coarsen.m,
# read_prolong.m, read_filter.m, read_general.m): one value per line, the first
# whitespace-separated token of each line; a '%' starts the trailing comment.
# ----------------------------------------------------------------------------

def _tokens(path, n):
    out = []
    with open(path) as f:
        for line in f:
            if len(out) == n:
                break
            tok = line.split()
            out.append(tok[0] if tok else "")
    if len(out) < n:
        raise ValueError(f"{path}: expected {n} lines, found {len(out)}")
    return out


def read_params(fnames_path):
    """readDefaultParams.m / aspAMG_main.m:17-59 restated."""
    d = os.path.dirname(os.path.abspath(fnames_path))
    names = _tokens(fnames_path, 7)
    p = lambda k: os.path.join(d, names[k])
    amg = _tokens(p(0), 2)
    smo = _tokens(p(1), 7)
    tsp = _tokens(p(2), 5)
    coa = _tokens(p(3), 3)
    pro = _tokens(p(4), 22)
    fil = _tokens(p(5), 5)
    gen = _tokens(p(6), 7)
    return {
        "amg": {"nLevMax": int(float(amg[0])), "maxCoarseSZ": int(float(amg[1]))},
        "smoother": {"nthread": int(float(smo[0])), "nupre": int(float(smo[1])),
                     "nupost": int(float(smo[2])), "nstep": int(float(smo[3])),
                     "step_size": int(float(smo[4])), "epsilon": float(smo[5]),
                     "method": smo[6]},
        "tspace": {"ntv": int(float(tsp[0])), "itmax": int(float(tsp[1])),
                   "tol": float(tsp[2]), "method": tsp[3], "init_approx": int(float(tsp[4]))},
        "coarsen": {"SoC_type": coa[0], "tau": float(coa[1]), "nl_agg": int(float(coa[2]))},
        "prolong": {"proltype": pro[0], "prol_emin": pro[1], "np": int(float(pro[2])),
                    "itmax_Vol": int(float(pro[3])), "tol_Vol": float(pro[4]),
                    "dist_min": int(float(pro[5])), "dist_max": int(float(pro[6])),
                    "maxcond": float(pro[7]), "maxrownrm": float(pro[8]),
                    "eps_prol": float(pro[9]), "updateCF": int(float(pro[10])),
                    "patt_pow": int(float(pro[11])), "patt_tau": float(pro[12]),
                    "nnzr_max": int(float(pro[13])), "itmax_emin": int(float(pro[14])),
                    "energ_tol": float(pro[15]), "condmax_emin": float(pro[16]),
                    "prec_emin": int(float(pro[17])), "solv_emin": int(float(pro[18]))},
        "filter": {"np": int(float(fil[0])), "filt_wgt": float(fil[1]),
                   "filt_tol": float(fil[2]), "filt_tau": float(fil[3]),
                   "min_patt": int(float(fil[4]))},
        "general": {"ascii_input": gen[0].lower() == "true", "rhs_build": gen[1],
                    "symmetric": gen[2].lower() == "true", "solv_method": gen[3],
                    "itmax": int(float(gen[4])), "tol": float(gen[5]),
                    "restart": int(float(gen[6]))},
    }


def default_params(nthread=None):
    """The reference's regression-test parameter set (Tests/parm_*)."""
    nthread = nthread or os.cpu_count() or 1
    return {
        "amg": {"nLevMax": 10, "maxCoarseSZ": 1000},
        "smoother": {"nthread": nthread, "nupre": 1, "nupost": 1, "nstep": 15,
                     "step_size": 1, "epsilon": 1e-3, "method": "AFSAI_SYM"},
        "tspace": {"ntv": 6, "itmax": 40, "tol": 1e-4, "method": "NONE", "init_approx": 5},
        "coarsen": {"SoC_type": "DOM", "tau": 0.01, "nl_agg": 0},
        "prolong": {"proltype": "BAMG", "prol_emin": "NONE", "np": nthread,
                    "itmax_Vol": 100, "tol_Vol": 0.01, "dist_min": 1, "dist_max": 10,
                    "maxcond": 1e13, "maxrownrm": 5.0, "eps_prol": 1e-10, "updateCF": 0,
                    "patt_pow": 2, "patt_tau": 0.01, "nnzr_max": 30, "itmax_emin": 10,
                    "energ_tol": 1e-3, "condmax_emin": 1e10, "prec_emin": 1, "solv_emin": 4},
        "filter": {"np": nthread, "filt_wgt": 170.0, "filt_tol": 0.1, "filt_tau": 0.0,
                   "min_patt": 0},
        "general": {"ascii_input": False, "rhs_build": "unit_rhs", "symmetric": True,
                    "solv_method": "PCG", "itmax": 15000, "tol": 1e-8, "restart": 100},
    }


# ----------------------------------------------------------------------------
# Fixture readers
# ----------------------------------------------------------------------------

def read_bin_matrix(path, ncols=None):
    """Binary COO of Cpp_EMIN/readMat.cpp:4-80: header {int32 nr, int32 nt},
    then nt records {int32 i, int32 j, float64 a}, 1-based, row-sorted."""
    with open(path, "rb") as f:
        nr, nt = np.frombuffer(f.read(8), dtype=np.int32)
        rec = np.frombuffer(f.read(16 * int(nt)),
                            dtype=np.dtype([("i", "<i4"), ("j", "<i4"), ("a", "<f8")]))
    i = rec["i"].astype(np.int64) - 1
    j = rec["j"].astype(np.int64) - 1
    nc = int(ncols) if ncols is not None else int(max(nr, j.max() + 1))
    return sp.csr_matrix((rec["a"].copy(), (i, j)), shape=(int(nr), nc))


def read_fcnode(path):
    return np.loadtxt(path, dtype=np.int64)


def read_tv(path):
    with open(path) as f:
        n, k = (int(t) for t in f.readline().split())
        data = np.loadtxt(f)
    return data.reshape(n, k)


def load_mat(path):
    return scipy.io.loadmat(path)


# ----------------------------------------------------------------------------
# MATLAB-compatible random stream (rng(0) -> MT19937 init_genrand(5489))
# ----------------------------------------------------------------------------

class MatlabRand:
    def __init__(self, seed=5489):
        self._rs = np.random.RandomState(seed)

    def rand(self, n, k=1):
        """rand(n,k): column-major fill of 53-bit doubles."""
        v = self._rs.random_sample(n * k)
        return v.reshape(k, n).T.copy() if k > 1 else v


# ----------------------------------------------------------------------------
# Reference C++ kernels through oracle/_ref
# ----------------------------------------------------------------------------

_libs = {}


def _ref_lib(name):
    if name not in _libs:
        path = os.path.join(REF_DIR, f"libref_{name}.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle ref`")
        _libs[name] = ctypes.CDLL(path)
    return _libs[name]


def ref_available():
    return all(os.path.exists(os.path.join(REF_DIR, f"libref_{n}.so"))
               for n in ("fsai", "bamg", "emin"))


def _ptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def ref_afsai(A, nthread, nstep, step_size, eps):
    """afsai_cpp.m:23-63 + SYM_aFSAI_compute: returns (F lower-triangular CSR,
    is_posdef).  Runs the reference's compute_local_fsai."""
    A = sp.csr_matrix(A)
    A.sort_indices()
    n = A.shape[0]
    iat = (A.indptr.astype(np.int64) + 1)
    ja = (A.indices.astype(np.int32) + 1)
    coef = np.ascontiguousarray(A.data, dtype=np.float64)
    kmax = 1 + nstep * step_size
    iat_G = np.zeros(n + 1, dtype=np.int64)
    ja_G = np.zeros(n * kmax, dtype=np.int32)
    coef_G = np.zeros(n * kmax, dtype=np.float64)
    nterm = np.zeros(1, dtype=np.int64)
    posdef = ctypes.c_int(0)
    lib = _ref_lib("fsai")
    lib.ref_fsai(ctypes.c_int(nthread), ctypes.c_int(nstep), ctypes.c_int(step_size),
                 ctypes.c_double(eps), ctypes.c_int(n), ctypes.c_int64(A.nnz),
                 _ptr(iat, ctypes.c_int64), _ptr(ja, ctypes.c_int),
                 _ptr(coef, ctypes.c_double), _ptr(nterm, ctypes.c_int64),
                 _ptr(iat_G, ctypes.c_int64), _ptr(ja_G, ctypes.c_int),
                 _ptr(coef_G, ctypes.c_double), ctypes.byref(posdef))
    nt = int(nterm[0])
    indptr = iat_G - 1
    # Rows keep the reference's order: strictly-lower entries ascending, the
    # diagonal last (cpt_afsai_coef.cpp:525-535).
    F = sp.csr_matrix((coef_G[:nt].copy(), ja_G[:nt].astype(np.int64) - 1, indptr),
                      shape=(n, n))
    return F, bool(posdef.value)


class _BamgResult(ctypes.Structure):
    _fields_ = [("nt", ctypes.c_int), ("iat", ctypes.POINTER(ctypes.c_int)),
                ("ja", ctypes.POINTER(ctypes.c_int)),
                ("coef", ctypes.POINTER(ctypes.c_double)),
                ("c_mark", ctypes.POINTER(ctypes.c_int))]


def ref_bamg(prm, nc, fcnode, S, TV):
    """cpt_ProlMEX_BAMG.m:33-66 restated; BAMG itself is the reference's C++.
    Returns (P csr n x nc with exact zeros dropped, c_mark)."""
    S = sp.csr_matrix(S)
    S.sort_indices()
    n = S.shape[0]
    fc = np.where(fcnode > 0, fcnode - 1, -1).astype(np.int32)
    TVr = np.ascontiguousarray(TV, dtype=np.float64)
    ntv = TVr.shape[1]
    iat = S.indptr.astype(np.int32)
    ja = S.indices.astype(np.int32)
    res = _BamgResult()
    lib = _ref_lib("bamg")
    ierr = lib.ref_bamg(ctypes.c_int(prm["np"]), ctypes.c_int(prm["itmax_Vol"]),
                        ctypes.c_int(prm["dist_min"]), ctypes.c_int(prm["dist_max"]),
                        ctypes.c_int(ntv), ctypes.c_double(prm["maxcond"]),
                        ctypes.c_double(prm["maxrownrm"]), ctypes.c_double(prm["tol_Vol"]),
                        ctypes.c_double(prm["eps_prol"]), ctypes.c_int(n),
                        _ptr(iat, ctypes.c_int), _ptr(ja, ctypes.c_int), ctypes.c_int(ntv),
                        _ptr(fc, ctypes.c_int), _ptr(TVr, ctypes.c_double), ctypes.byref(res))
    if ierr != 0:
        raise RuntimeError(f"reference BAMG failed with code {ierr}")
    nt = res.nt
    indptr = np.ctypeslib.as_array(res.iat, shape=(n + 1,)).astype(np.int64).copy()
    cols = np.ctypeslib.as_array(res.ja, shape=(max(nt, 1),))[:nt].astype(np.int64).copy()
    vals = np.ctypeslib.as_array(res.coef, shape=(max(nt, 1),))[:nt].copy()
    c_mark = np.ctypeslib.as_array(res.c_mark, shape=(n,)).copy()
    lib.ref_bamg_free(ctypes.byref(res))
    P = sp.csr_matrix((vals, cols, indptr), shape=(n, nc))
    P.eliminate_zeros()      # the MEX gateway skips explicit zeros (gateway :131-137)
    P.sort_indices()
    return P, c_mark


class _RefCsr(ctypes.Structure):
    _fields_ = [("nrows", ctypes.c_int), ("ncols", ctypes.c_int), ("nnz", ctypes.c_int),
                ("rp", ctypes.POINTER(ctypes.c_int)), ("ci", ctypes.POINTER(ctypes.c_int)),
                ("v", ctypes.POINTER(ctypes.c_double))]


def _csr32(M):
    M = sp.csr_matrix(M)
    M.sort_indices()
    return (M, M.indptr.astype(np.int32), M.indices.astype(np.int32),
            np.ascontiguousarray(M.data, dtype=np.float64))


def _take_ref_csr(lib, res):
    m, nnz = res.nrows, res.nnz
    rp = np.ctypeslib.as_array(res.rp, shape=(m + 1,)).astype(np.int64).copy()
    ci = np.ctypeslib.as_array(res.ci, shape=(max(nnz, 1),))[:nnz].astype(np.int64).copy()
    v = np.ctypeslib.as_array(res.v, shape=(max(nnz, 1),))[:nnz].copy()
    shape = (m, res.ncols)
    lib.ref_csr_free(ctypes.byref(res))
    return sp.csr_matrix((v, ci, rp), shape=shape)


def _fc_c(fcnode):
    """MATLAB fcnode (coarse index + 1 > 0, fine < 0) -> the C++ convention of
    MEX_EMIN_enhance_prol.m:73 (coarse index >= 0, fine < 0)."""
    return np.where(np.asarray(fcnode) > 0, np.asarray(fcnode) - 1, -1).astype(np.int32)


def ref_emin_pattern(kpow, S, P, fcnode, nnzr, nnzr_min, np_threads=1):
    """MEX_cptProlPatt (the reference's C++, oracle/_ref) as prolong.m:222 calls
    it; fcnode in MATLAB's convention.  Returns the n x nc pattern (CSR with the
    values the MEX returns: 1 on P's own entries, S*P's on the added ones)."""
    S, sr, sc, sv = _csr32(S)
    P, pr_, pc, pv = _csr32(P)
    n, nc = P.shape
    fc = _fc_c(fcnode)
    res = _RefCsr()
    lib = _ref_lib("emin")
    rc = lib.ref_emin_pattern(ctypes.c_int(kpow), ctypes.c_int(n), ctypes.c_int(nc),
                              _ptr(sr, ctypes.c_int), _ptr(sc, ctypes.c_int),
                              _ptr(sv, ctypes.c_double), _ptr(pr_, ctypes.c_int),
                              _ptr(pc, ctypes.c_int), _ptr(pv, ctypes.c_double),
                              _ptr(fc, ctypes.c_int), ctypes.c_int(nnzr), ctypes.c_int(nnzr_min),
                              ctypes.c_int(np_threads), ctypes.byref(res))
    if rc != 0:
        raise RuntimeError("reference MEX_cptProlPatt raised an error")
    return _take_ref_csr(lib, res)


def ref_emin(prm, A, Ppatt, P, TV, fcnode, spd=True):
    """EMIN_ImpProl (the reference's C++, oracle/_ref) with the arguments of
    MEX_EMIN_enhance_prol.m:29-98; fcnode in MATLAB's convention.  Returns
    (P, info) with P's exact zeros dropped as sparse() does there (:102)."""
    A, ar, ac, av = _csr32(A)
    P, pr_, pc, pv = _csr32(P)
    Pp, tr, tc, _ = _csr32(Ppatt)
    n, nc = P.shape
    TVr = np.ascontiguousarray(TV, dtype=np.float64)
    fc = _fc_c(fcnode)
    res = _RefCsr()
    info = np.zeros(12)
    lib = _ref_lib("emin")
    ierr = lib.ref_emin(ctypes.c_int(prm["np"]), ctypes.c_int(prm["itmax_emin"]),
                        ctypes.c_double(prm["energ_tol"]), ctypes.c_double(prm["condmax_emin"]),
                        ctypes.c_int(prm["prec_emin"]), ctypes.c_int(prm["solv_emin"]),
                        ctypes.c_int(n), ctypes.c_int(nc), ctypes.c_int(TVr.shape[1]),
                        _ptr(fc, ctypes.c_int), ctypes.c_int(1 if spd else 0),
                        _ptr(ar, ctypes.c_int), _ptr(ac, ctypes.c_int), _ptr(av, ctypes.c_double),
                        _ptr(pr_, ctypes.c_int), _ptr(pc, ctypes.c_int), _ptr(pv, ctypes.c_double),
                        _ptr(tr, ctypes.c_int), _ptr(tc, ctypes.c_int),
                        _ptr(TVr, ctypes.c_double), ctypes.byref(res),
                        _ptr(info, ctypes.c_double))
    if ierr != 0:
        raise RuntimeError(f"reference EMIN failed with code {ierr}")
    Pout = _take_ref_csr(lib, res)
    Pout.eliminate_zeros()
    Pout.sort_indices()
    return Pout, info


# ----------------------------------------------------------------------------
# Coarsening (host code of the reference; restated)
# ----------------------------------------------------------------------------

def mark_isolated_nodes(A, fcnode):
    """mark_isolated_nodes.m:1-8: nodes whose column holds one nonzero -> -2."""
    coo = sp.coo_matrix(A)
    nz = coo.data != 0
    col_counts = np.bincount(coo.col[nz], minlength=A.shape[1])
    iso = np.flatnonzero(col_counts == 1)
    fcnode = fcnode.copy()
    fcnode[iso] = -2
    return fcnode, iso.size


def soc_dom(tau, A):
    """cpt_SoC_dom.m:25-63 (tau >= 0 branch): s_ij = |a_ij|/sqrt(a_ii a_jj),
    strong when s_ij > tau (diagonal included, s_ii = 1)."""
    A = sp.coo_matrix(A)
    keep = A.data != 0
    ii, jj, aa = A.row[keep], A.col[keep], A.data[keep]
    dd = sp.csr_matrix(A).diagonal()
    ss = np.abs(aa) / np.sqrt(dd[ii] * dd[jj])
    if tau < 0:
        raise NotImplementedError("negative tau (average-count filter) is not part of this path")
    n = A.shape[0]
    sf = np.where(ss > tau, ss, 0.0)
    S = sp.csr_matrix((sf, (ii, jj)), shape=(n, n))
    S.eliminate_zeros()
    S.sort_indices()
    return S


def soc_cla(tau, A):
    """cpt_SoC_cla.m:107-159: classical M-matrix strength with the
    absolute-value fallback, then S + I."""
    A = sp.csr_matrix(A)
    n = A.shape[0]
    d = A.diagonal()
    A_off = (A - sp.diags(d)).tocsc()
    A_off.eliminate_zeros()
    # min over each column including implicit zeros (MATLAB min of a sparse column)
    min_col = np.zeros(n)
    cnt = np.diff(A_off.indptr)
    for j in range(n):
        seg = A_off.data[A_off.indptr[j]:A_off.indptr[j + 1]]
        m = seg.min() if seg.size else 0.0
        min_col[j] = min(m, 0.0) if cnt[j] < n else m
    Ac = sp.coo_matrix(A)
    keep = Ac.data != 0
    ii, jj, aa = Ac.row[keep], Ac.col[keep], Ac.data[keep]
    if np.all(min_col >= 0):
        max_abs = np.zeros(n)
        for j in range(n):
            seg = np.abs(A_off.data[A_off.indptr[j]:A_off.indptr[j + 1]])
            max_abs[j] = seg.max() if seg.size else 0.0
        max_abs[max_abs == 0] = 1.0
        ss = np.abs(aa) / np.maximum(max_abs[ii], max_abs[jj])
    else:
        min_col[min_col == 0] = 1.0
        ss = aa / np.maximum(min_col[ii], min_col[jj])
    sf = np.where(ss > tau, ss, 0.0)
    S = sp.csr_matrix((sf, (ii, jj)), shape=(n, n))
    S.eliminate_zeros()
    S = (S + sp.identity(n, format="csr")).tocsr()
    S.sort_indices()
    return S


def cpt_pmis(S, fcnode, rng):
    """cpt_PMIS.m:1-102, sequential list sweep exactly as the reference.
    fcnode: 0 free, -2 Dirichlet.  Returns 1-based-numbered fcnode
    (coarse k = 1..nc, fine -(1..nf)), clist, flist (0-based indices)."""
    S = sp.csr_matrix(S, copy=True)
    nn = S.shape[0]
    S.setdiag(0)
    S.eliminate_zeros()
    Sc = S.tocsc()
    Sc.sort_indices()
    S_sym = (abs(S) + abs(S.T)).tocsc()
    S_sym.eliminate_zeros()
    S_sym.sort_indices()
    nod_weight = np.diff(Sc.indptr).astype(np.float64)        # sum(S ~= 0, 1)'
    fcnode = fcnode.copy()
    fcnode[fcnode == -2] = -1
    nod_weight = nod_weight + rng.rand(nn)
    w_free = nod_weight.copy()
    w_free[fcnode == -1] = -1.0
    lst = list(np.flatnonzero(fcnode == 0))
    len_list = len(lst)
    ind = 0
    sp_ptr, sp_idx = S_sym.indptr, S_sym.indices
    sc_ptr, sc_idx = Sc.indptr, Sc.indices
    while len_list > 0:
        inod = lst[ind]
        if fcnode[inod] != 0:
            lst[ind] = lst[len_list - 1]
            len_list -= 1
        else:
            is_coarse = True
            w = nod_weight[inod]
            nb = sp_idx[sp_ptr[inod]:sp_ptr[inod + 1]]
            if nb.size and np.any(w_free[nb] > w):
                is_coarse = False
                ind += 1
            if is_coarse:
                nb2 = sc_idx[sc_ptr[inod]:sc_ptr[inod + 1]]
                fcnode[nb2] = -1
                w_free[nb2] = -1.0
                fcnode[inod] = 1
                w_free[inod] = -1.0
                lst[ind] = lst[len_list - 1]
                len_list -= 1
        if ind > len_list - 1:
            ind = 0
    clist = np.flatnonzero(fcnode > 0)
    flist = np.flatnonzero(fcnode < 0)
    fcnode[clist] = np.arange(1, clist.size + 1)
    fcnode[flist] = -np.arange(1, flist.size + 1)
    return fcnode, clist, flist


def coarsen(prm, A, rng):
    """coarsen.m:30-76 for the SoC types on this path (DOM, CLA)."""
    n = A.shape[0]
    fcnode, _ = mark_isolated_nodes(A, np.zeros(n, dtype=np.int64))
    t = prm["SoC_type"].upper()
    if t == "DOM":
        S = soc_dom(prm["tau"], A)
    elif t == "CLA":
        S = soc_cla(prm["tau"], A)
    else:
        raise NotImplementedError(f"SoC type {t} is outside this path")
    fcnode, clist, flist = cpt_pmis(S, fcnode, rng)
    return fcnode, clist, flist, S


# ----------------------------------------------------------------------------
# Hierarchy (cpt_aspAMG.m) and its application (AMG_Vcycle.m)
# ----------------------------------------------------------------------------

@dataclass
class Level:
    A: sp.csr_matrix
    G: sp.csr_matrix | None = None      # FSAI factor F (lower triangular)
    omega: float = 1.0
    P: sp.csr_matrix | None = None
    fcnode: np.ndarray | None = None
    L: np.ndarray | None = None         # coarsest dense Cholesky factor
    nupre: int = 1
    nupost: int = 1
    lam: float = 0.0


@dataclass
class Hierarchy:
    levels: list = field(default_factory=list)


def smoother_afsai(A, prm):
    """smoother.m:33-87 (afsai_sym branch, SPD)."""
    F, posdef = ref_afsai(A, prm["nthread"], prm["nstep"], prm["step_size"], prm["epsilon"])
    if not posdef:
        raise RuntimeError("FSAI: matrix deemed indefinite (NSY fallback is outside this path)")
    d = F.diagonal()
    bad = np.flatnonzero(np.isnan(d))
    if bad.size:
        F = F.tolil()
        dA = A.diagonal()
        for i in bad:
            F[i, :] = 0
            F[i, i] = 1.0 / np.sqrt(dA[i])
        F = F.tocsr()
    lam = lambda_max_fsai(A, F)
    return F, min(1.0, 1.9 / lam), lam


def lambda_max_fsai(A, F, tol=5e-4):
    """eigs(F*A*F','la',opts.tol=5e-4) (smoother.m:73-77) via ARPACK."""
    n = A.shape[0]
    Ft = F.T.tocsr()
    op = spla.LinearOperator((n, n), matvec=lambda x: F @ (A @ (Ft @ x)), dtype=np.float64)
    v0 = np.ones(n) / np.sqrt(n)
    lam = spla.eigsh(op, k=1, which="LA", tol=tol, v0=v0, return_eigenvectors=False)
    return float(lam[0])


def galerkin(P, A):
    """Anext = Pf'*(A*Pf) (cpt_aspAMG.m:277): two Gustavson products, exact
    zeros dropped after each (scipy csr_matmat, as MATLAB's sparse product)."""
    AP = (A @ P).tocsr()
    AP.eliminate_zeros()
    Pt = P.T.tocsr()
    Pt.sort_indices()
    Ac = (Pt @ AP).tocsr()
    Ac.eliminate_zeros()
    Ac.sort_indices()
    return Ac


def qr_thin(TV):
    Q, _ = np.linalg.qr(TV, mode="reduced")
    return Q


def cpt_aspamg(param, A, TV0, rng=None, on_level=None):
    """cpt_aspAMG.m:1-64 + REC_cpt_aspAMG :68-351 for the SPD path (filters
    off: filt_wgt >= 100 and filt_tau = 0)."""
    rng = rng or MatlabRand()
    A = sp.csr_matrix(A)
    A.sort_indices()
    n = A.shape[0]
    ntv = param["tspace"]["ntv"]
    TV0 = np.zeros((n, 0)) if TV0 is None else np.asarray(TV0, dtype=np.float64).reshape(n, -1)
    ntv0 = TV0.shape[1]
    TV = np.zeros((n, ntv))
    if ntv0 > 0:
        ncol = min(ntv0, ntv)
        TV[:, :ncol] = TV0[:, :ncol]
    if ntv > ntv0:
        TV[:, ntv0:ntv] = rng.rand(n, ntv - ntv0).reshape(n, ntv - ntv0)
    TV = qr_thin(TV)
    hier = Hierarchy()
    level = 0
    if param["filter"]["filt_wgt"] < 100 or param["filter"]["filt_tau"] > 0:
        raise NotImplementedError("prolongation / coarse-operator filters are outside this path")
    while True:
        level += 1
        n = A.shape[0]
        if n <= param["amg"]["maxCoarseSZ"] or level >= param["amg"]["nLevMax"]:
            L = np.linalg.cholesky(A.toarray())
            hier.levels.append(Level(A=A, L=L))
            break
        G, omega, lam = smoother_afsai(A, param["smoother"])
        TV = qr_thin(TV)                                   # tspace NONE (tspace.m:51-55)
        fcnode, clist, flist, S = coarsen(param["coarsen"], A, rng)
        if param["prolong"]["proltype"].upper() != "BAMG":
            raise NotImplementedError("only BAMG prolongation is on this path")
        P, c_mark = ref_bamg(param["prolong"], clist.size, fcnode, S, TV)
        emin = param["prolong"].get("prol_emin", "NONE").upper()
        if emin == "SMOOTH":
            P = smooth_prolongation(A, P)
        elif emin == "EMIN":
            P = emin_reference(param, A, S, P, TV, fcnode)
        elif emin != "NONE":
            raise NotImplementedError("prolongation post-process " + emin)
        TV = TV[clist, :]
        Ac = galerkin(P, A)
        lev = Level(A=A, G=G, omega=omega, P=P, fcnode=fcnode,
                    nupre=param["smoother"]["nupre"], nupost=param["smoother"]["nupost"], lam=lam)
        hier.levels.append(lev)
        if on_level:
            on_level(level, lev)
        A = Ac
    return hier


def emin_reference(param, A, S, P, TV, fcnode):
    """prolong.m:207-235 with the reference's own C++ (oracle/_ref): S_emin is
    the coarsening's S when it is DOM with tau = patt_tau, else
    cpt_SoC_dom(patt_tau, A); Ppatt = MEX_cptProlPatt(patt_pow, S_emin, P,
    fcnode, nnzr_max, ntv, np); P = MEX_EMIN_enhance_prol(...)."""
    pro, coa = param["prolong"], param["coarsen"]
    if coa["SoC_type"].upper() == "DOM" and coa["tau"] == pro["patt_tau"]:
        S_emin = S
    else:
        S_emin = soc_dom(pro["patt_tau"], A)
    ntv = np.asarray(TV).shape[1]
    Ppatt = ref_emin_pattern(pro["patt_pow"], S_emin, P, fcnode, pro["nnzr_max"], ntv,
                             pro["np"])
    Pe, _ = ref_emin(pro, A, Ppatt, P, TV, fcnode)
    return Pe


def hierarchy_from_parts(parts, nupre=1, nupost=1):
    """Oracle hierarchy from given per-level matrices: parts is a list of dicts
    with A, G, omega, P (all levels but the last) and A alone for the last,
    whose dense Cholesky factor is computed here (FP64)."""
    H = Hierarchy()
    for k, p in enumerate(parts):
        A = sp.csr_matrix(p["A"])
        if k == len(parts) - 1:
            H.levels.append(Level(A=A, L=np.linalg.cholesky(A.toarray())))
        else:
            H.levels.append(Level(A=A, G=sp.csr_matrix(p["G"]), omega=float(p["omega"]),
                                  P=sp.csr_matrix(p["P"]), nupre=nupre, nupost=nupost))
    return H


def amg_vcycle(hier, b, lvl=0, A=None):
    """AMG_Vcycle.m:1-54 (no x0)."""
    lev = hier.levels[lvl]
    A = lev.A if A is None else A
    if lev.L is not None:
        y = scipy.linalg.solve_triangular(lev.L, b, lower=True)
        return scipy.linalg.solve_triangular(lev.L.T, y, lower=False)
    G, Gt, w = lev.G, lev.G.T, lev.omega
    x = w * (Gt @ (G @ b))
    for _ in range(1, lev.nupre):
        r = b - A @ x
        x = x + w * (Gt @ (G @ r))
    r = b - A @ x
    rc = lev.P.T @ r
    hc = amg_vcycle(hier, rc, lvl + 1)
    x = x + lev.P @ hc
    for _ in range(lev.nupost):
        r = b - A @ x
        x = x + w * (Gt @ (G @ r))
    return x


def pcg_cj(prodM, prodA, b, x0, itmax, tol):
    """PCG_CJ.m:1-73, same recurrence and stopping test."""
    nn = b.shape[0]
    it = 0
    flag = 0
    resvec = np.zeros(max(itmax, 0) + 1)
    bnorm = np.linalg.norm(b)
    if bnorm == 0.0:
        return np.zeros(nn), 0, resvec[:1], 0
    x = x0.copy()
    res = b - prodA(x)
    resiter = np.linalg.norm(res) / bnorm
    resvec[0] = resiter
    exit_test = itmax <= 0
    p = axp = None
    ptap = 0.0
    while not exit_test:
        it += 1
        pres = prodM(res)
        if it == 1:
            p = pres.copy()
        else:
            beta = -(pres @ axp) / ptap
            p = pres + beta * p
        axp = prodA(p)
        ptap = p @ axp
        alpha = (p @ res) / ptap
        x = x + alpha * p
        res = res - alpha * axp
        resiter = np.linalg.norm(res) / bnorm
        resvec[it] = resiter
        exit_test = resiter < tol or it == itmax
    if resiter > tol:
        flag = 1
    return x, it, resvec[:it + 1], flag


def sqmr(Afun, rhs, tol, itmax, lprec, rprec=lambda v: v, x0=None):
    """SQMR.m:1-108; returns (x, info, relres, niter, resvec)."""
    nn = rhs.shape[0]
    d = np.zeros(nn)
    pnew = np.zeros(nn) if x0 is None else x0.copy()
    resvec = np.zeros(itmax)
    info = 0
    exit_test = False
    niter = 0
    bnorm = np.linalg.norm(rhs)
    r = rhs - Afun(pnew)
    vscr = lprec(r)
    q = rprec(vscr)
    tau = np.linalg.norm(vscr)
    rho0 = r @ q
    theta0 = 0.0
    while not exit_test and niter < itmax:
        niter += 1
        vscr = Afun(q)
        sigma = q @ vscr
        if abs(sigma) < 1e-20 * rho0:
            info = 10
            break
        alpha = rho0 / sigma
        r = r - alpha * vscr
        vscr = lprec(r)
        theta1 = np.linalg.norm(vscr) / tau
        gamma = 1.0 / np.sqrt(1.0 + theta1 * theta1)
        tau = tau * theta1 * gamma
        d = d * gamma * gamma * theta0 * theta0 + gamma * gamma * alpha * q
        theta0 = theta1
        pnew = pnew + d
        resnorm = np.linalg.norm(r) / bnorm
        if resnorm < tol:
            exit_test = True
        else:
            u = rprec(vscr)
            rho1 = r @ u
            if abs(rho0) < 1e-20 * rho1:
                info = 20
                break
            beta = rho1 / rho0
            rho0 = rho1
            q = u + beta * q
        resvec[niter - 1] = resnorm
    if niter >= itmax:
        info = 1
    relres = np.linalg.norm(rhs - Afun(pnew)) / bnorm
    return pnew, info, relres, niter, resvec[:niter]


def _sgn(v):
    """scalarsign: sign with sign(0) = 1."""
    return -1.0 if v < 0 else 1.0


def _solve_upper(R, y):
    """Solution of R z = y for upper-triangular R (back substitution)."""
    import scipy.linalg as sla
    return sla.solve_triangular(np.triu(R), y, lower=False)


def gmres_right(afun, b, restart, tol, maxit, mfun=None, x0=None):
    """Right-preconditioned restarted GMRES with Householder Arnoldi,
    restating gmres_RIGHT.m (LinearSolver/GMRES_CJ/gmres_RIGHT.m:7-650):
    inner iterations test the implicit residual |w(k+1)| <= tol*||b||
    (:398-409), confirm it with the explicit residual of x + inv(M) U y
    (:410-485), take up to maxmsteps more steps when it is not confirmed
    (:486-540), and restart from the iterate of minimal residual (:552-627).
    Returns (x, flag, relres, (outer, inner), resvec)."""
    n = b.shape[0]
    eps = np.finfo(float).eps
    M = mfun if mfun is not None else (lambda v: v)
    restart = max(int(restart), 0)
    outer, inner = max(int(maxit), 0), min(restart, n)                   # :143-157
    n2b = np.linalg.norm(b)
    if n2b == 0:                                                         # :160-172
        return np.zeros(n), 0, 0.0, (0, 0), np.zeros(1)
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=float)
    flag = 1
    xmin = x.copy()
    imin = jmin = 0
    tolb = tol * n2b
    evalxm = 0
    stag = 0
    moresteps = 0
    maxmsteps = min(n // 50, 5, n - maxit)                               # :221
    maxstagsteps = 3
    minupdated = 0
    r = b - afun(x)
    normr = np.linalg.norm(r)
    if normr <= tolb:                                                    # :226-237
        return x, 0, normr / n2b, (0, 0), np.array([normr])
    resvec = np.zeros(inner * outer + 1)
    resvec[0] = normr
    normrmin = normr
    J = np.zeros((2, inner))
    U = np.zeros((n, inner))
    R = np.zeros((inner, inner))
    w = np.zeros(inner + 1)
    it = (0, 0)
    outiter = initer = 0
    normr_act = normr
    xm = x

    def expand(y, k):
        """Product of the first k reflectors applied to y(1:k) (:412-418)."""
        add = U[:, k - 1] * (-2.0 * y[k - 1] * U[k - 1, k - 1])
        add[k - 1] += y[k - 1]
        for j in range(k - 1, 0, -1):
            add[j - 1] += y[j - 1]
            add = add - U[:, j - 1] * (2.0 * (U[:, j - 1] @ add))
        return add

    for outiter in range(1, outer + 1):
        u = r.copy()                                                     # :302-316
        normr = np.linalg.norm(r)
        beta = _sgn(r[0]) * normr
        u[0] += beta
        u = u / np.linalg.norm(u)
        U[:, 0] = u
        w[:] = 0.0
        w[0] = -beta
        for initer in range(1, inner + 1):
            v = -2.0 * u[initer - 1] * u                                 # :317-331
            v[initer - 1] += 1.0
            for k in range(initer - 1, 0, -1):
                v = v - U[:, k - 1] * (2.0 * (U[:, k - 1] @ v))
            v = M(v)                                                     # :332-352
            if not np.all(np.isfinite(v)):
                flag = 2
                break
            v = afun(v)
            for k in range(1, initer + 1):                               # :353-356
                v = v - U[:, k - 1] * (2.0 * (U[:, k - 1] @ v))
            if initer != n:                                              # :359-378
                u = v.copy()
                u[:initer] = 0.0
                alpha = np.linalg.norm(u)
                if alpha != 0:
                    alpha = _sgn(v[initer]) * alpha
                    u[initer] += alpha
                    u = u / np.linalg.norm(u)
                    if initer < inner:
                        U[:, initer] = u
                    v[initer + 1:] = 0.0
                    v[initer] = -alpha
            for c in range(initer - 1):                                  # :380-384
                tmp = v[c]
                v[c] = J[0, c] * v[c] + J[1, c] * v[c + 1]
                v[c + 1] = -J[1, c] * tmp + J[0, c] * v[c + 1]
            if initer != n:                                              # :387-395
                rho = np.linalg.norm(v[initer - 1:initer + 1])
                J[:, initer - 1] = v[initer - 1:initer + 1] / rho
                w[initer] = -J[1, initer - 1] * w[initer - 1]
                w[initer - 1] = J[0, initer - 1] * w[initer - 1]
                v[initer - 1] = rho
                v[initer] = 0.0
            R[:, initer - 1] = v[:inner]
            normr = abs(w[initer])                                       # :396-406
            resvec[(outiter - 1) * inner + initer] = normr
            normr_act = normr
            if normr <= tolb or stag >= maxstagsteps or moresteps:       # :409
                if evalxm == 0:                                          # :410-442
                    ytmp = _solve_upper(R[:initer, :initer], w[:initer])
                    add = expand(ytmp, initer)
                    stag = stag + 1 if np.linalg.norm(add) < eps * np.linalg.norm(x) else 0
                    add = M(add)
                    if not np.all(np.isfinite(add)):
                        flag = 2
                        break
                    xm = x + add
                    evalxm = 1
                else:                                                    # :443-476
                    Rk = np.triu(R[:initer, :initer])
                    last = w[initer - 1] / Rk[initer - 1, initer - 1]
                    head = (-_solve_upper(Rk[:initer - 1, :initer - 1],
                                          Rk[:initer - 1, initer - 1]) * last
                            if initer > 1 else np.zeros(0))
                    addvc = np.append(head, last)
                    stag = stag + 1 if np.linalg.norm(addvc) < eps * np.linalg.norm(xm) else 0
                    add = M(expand(addvc, initer))
                    if not np.all(np.isfinite(add)):
                        flag = 2
                        break
                    xm = xm + add
                r = b - afun(xm)                                         # :477-484
                if np.linalg.norm(r) <= tol * n2b:
                    x = xm
                    flag = 0
                    it = (outiter, initer)
                    break
                normr_act = np.linalg.norm(r)
                resvec[(outiter - 1) * inner + initer] = normr_act
                if normr_act <= normrmin:                                # :496-508
                    normrmin, imin, jmin, xmin, minupdated = normr_act, outiter, initer, xm, 1
                if normr_act <= tolb:
                    x = xm
                    flag = 0
                    it = (outiter, initer)
                    break
                if stag >= maxstagsteps and moresteps == 0:              # :515-531
                    stag = 0
                moresteps += 1
                if moresteps >= maxmsteps:
                    flag = 3
                    it = (outiter, initer)
                    break
            if normr_act <= normrmin:                                    # :534-545
                normrmin, imin, jmin, minupdated = normr_act, outiter, initer, 1
            if stag >= maxstagsteps:
                flag = 3
                break
        evalxm = 0                                                       # :552-627
        if flag != 0:
            idx = jmin if minupdated else initer
            if idx > 0:
                y = _solve_upper(R[:idx, :idx], w[:idx])
                add = M(expand(y, idx))
                if not np.all(np.isfinite(add)):
                    flag = 2
                    break
                x = x + add
            xmin = x
            r = b - afun(x)
            normr_act = np.linalg.norm(r)
        if normr_act <= normrmin:
            xmin, normrmin, imin, jmin = x, normr_act, outiter, initer
        if flag == 3:
            break
        if normr_act <= tolb:
            flag = 0
            it = (outiter, initer)
            break
        minupdated = 0
    relres = normr_act / n2b                                             # :637-644
    if flag != 0:
        x = xmin
        it = (imin, jmin)
    resvec = resvec[:max(outiter - 1, 0) * inner + initer + 1]           # :645-648
    if flag == 2 and initer != 0:
        resvec = resvec[:-1]
    return x, flag, relres, it, resvec


def smooth_prolongation(A, P, tol=1e-3):
    """prolong.m:180-196 (prol_emin = SMOOTH): DA = diag(diag(A))\\A (each row
    divided by its diagonal entry), lambda_max = eigs(DA,1,'lm') with
    tolerance 1e-3, omega = 1.9/lambda_max, P - omega*DA*P evaluated as
    (omega*DA)*P; MATLAB's sparse results drop exact zeros."""
    A = sp.csr_matrix(A)
    d = A.diagonal()
    DA = A.copy().astype(np.float64)
    DA.data = DA.data / np.repeat(d, np.diff(DA.indptr))
    n = A.shape[0]
    v0 = np.ones(n) / np.sqrt(n)
    try:
        lam = spla.eigs(DA, k=1, which="LM", tol=tol, v0=v0, return_eigenvectors=False,
                        maxiter=max(3 * n, 1000))
    except spla.ArpackNoConvergence as e:
        lam = e.eigenvalues
    omega = 1.9 / float(abs(lam[0]))
    W = DA.copy()
    W.data = omega * W.data
    WP = (W @ sp.csr_matrix(P)).tocsr()
    Ps = (sp.csr_matrix(P) - WP).tocsr()
    Ps.eliminate_zeros()
    Ps.sort_indices()
    return Ps


def emin_pattern(kpow, S, P, fcnode, nnzr_max, nnzr_min):
    """MEX_cptProlPatt.cpp:234-490 restated (prolong.m:222 passes kpow =
    patt_pow, nnzr_min = ntv).  fcnode in MATLAB's convention.  Each power
    step lists, per row i, the columns of (S * P_cur)(i, :) outside P's own
    row in first-seen order (S's row order, then P_cur's), with values summed
    in that order; keeps the nonzero ones; when there are more than the budget
    nnzr - |P(i,:)|, keeps the budget's worth of largest |value| (ties: lower
    column first); adds P's own columns with value 1; sorts by column.  Coarse
    rows are empty after the last step.  kpow <= 1 keeps P's fine rows."""
    P0 = sp.csr_matrix(P)
    P0.sort_indices()
    S = sp.csr_matrix(S)
    S.sort_indices()
    n, nc = P0.shape
    fcnode = np.asarray(fcnode)
    nnzr = max(nnzr_max, nnzr_min)
    if kpow <= 1:
        keep = np.repeat(fcnode <= 0, np.diff(P0.indptr))
        rows = np.repeat(np.arange(n), np.diff(P0.indptr))[keep]
        return sp.csr_matrix((P0.data[keep], (rows, P0.indices[keep])), shape=(n, nc))
    Pc = P0
    for ipow in range(2, kpow + 1):
        last = ipow == kpow
        indptr, cols, vals = [0], [], []
        for i in range(n):
            if last and fcnode[i] > 0:
                indptr.append(len(cols))
                continue
            own = P0.indices[P0.indptr[i]:P0.indptr[i + 1]]
            budget = max(0, nnzr - own.size)
            if budget == 0:
                cols.extend(own.tolist())
                vals.extend([1.0] * own.size)
                indptr.append(len(cols))
                continue
            own_set = set(own.tolist())
            acc = {}
            for ks in range(S.indptr[i], S.indptr[i + 1]):
                j, sij = S.indices[ks], S.data[ks]
                for kp in range(Pc.indptr[j], Pc.indptr[j + 1]):
                    c = int(Pc.indices[kp])
                    if c in own_set:
                        continue
                    if c in acc:
                        acc[c] = acc[c] + sij * Pc.data[kp]
                    else:
                        acc[c] = sij * Pc.data[kp]
            cand = [(c, v) for c, v in acc.items() if v != 0.0]
            if len(cand) > budget:
                cand = sorted(cand, key=lambda cv: (-abs(cv[1]), cv[0]))[:budget]
            cand += [(int(c), 1.0) for c in own]
            cand.sort(key=lambda cv: cv[0])
            cols.extend(c for c, _ in cand)
            vals.extend(v for _, v in cand)
            indptr.append(len(cols))
        Pc = sp.csr_matrix((np.array(vals, dtype=np.float64), np.array(cols, dtype=np.int64),
                            np.array(indptr, dtype=np.int64)), shape=(n, nc))
    return Pc


def _orth_q(Q, nr, x):
    """Orth_Q.cpp:6-74 for one row block: x - Q (Q' x)."""
    return x - Q @ (Q.T @ x)


def emin_enhance(prm, A, Ppatt, P, TV, fcnode):
    """EMIN_matfree.cpp:69-308 with solv_emin = 4 (SPMAT), prec_emin = 1
    (Jacobi) and an SPD A, restated.  fcnode in MATLAB's convention; Ppatt's
    coarse rows are empty (MEX_cptProlPatt).  Unknowns are P's fine-row
    entries on the pattern, row-major.  Steps:

      copy_Prol.cpp:7-53       P0 = P on the pattern (zero where P has none)
      gather_B_QR.cpp:33-587   per fine row i with pattern columns c_1..c_m,
                               B = TV(coarse nodes c_k, :) (m x ntv);
                               g = TV(i,:)' - B' p0; m > ntv and
                               max|R_kk|/min|R_kk| <= condmax: Householder QR,
                               p0 += Q R^-T g, keep Q; otherwise thin SVD,
                               rank = 1 + #{k >= 1: s_0 < condmax |s_k|}
                               (0 if s_0 <= 1e-15), p0 += U_r S_r^-1 V_r' g,
                               keep [U_r, 0]
      gather_f.cpp:1-50        f(i,c) = -A(c, i) on the pattern
      cpt_Trace_Acc.cpp:4-18   Tr_A = sum of A's diagonal over coarse nodes
      load_Jacobi.cpp:4-21     D(i,c) = 1/A(i,i) (1 when |A(i,i)| <= 1e-15)
      KP_spmat.cpp:11-73       K x = (A X)|pattern, X = x on the fine rows
      DEFL_PCG_matfree.cpp     projected PCG on K d = K p0 - f, projector
                               I - Q Q' per row, Jacobi preconditioner, at
                               most itmax_emin steps, stop when the step's
                               energy decrease falls below energ_tol times
                               the first step's; P = P0 - d
      Prol_add_Cnodes.cpp      coarse rows: identity entries

    Returns (P n x nc with exact zeros dropped, iterations)."""
    A = sp.csr_matrix(A)
    A.sort_indices()
    Pp = sp.csr_matrix(Ppatt)
    Pp.sort_indices()
    Pin = sp.csr_matrix(P)
    Pin.sort_indices()
    n, nc = Pin.shape
    TV = np.asarray(TV, dtype=np.float64)
    ntv = TV.shape[1]
    fcnode = np.asarray(fcnode)
    coarse = fcnode > 0
    c2glo = np.flatnonzero(coarse)[np.argsort(fcnode[coarse])]
    rp, ci = Pp.indptr, Pp.indices
    nt = int(rp[n])
    rows = np.repeat(np.arange(n), np.diff(rp))
    # copy_Prol
    p0 = np.zeros(nt)
    for i in np.flatnonzero(~coarse):
        pos = {int(c): k for k, c in enumerate(ci[rp[i]:rp[i + 1]], start=rp[i])}
        for k in range(Pin.indptr[i], Pin.indptr[i + 1]):
            kk = pos.get(int(Pin.indices[k]))
            if kk is not None:
                p0[kk] = Pin.data[k]
    # gather_B_QR
    condmax = prm["condmax_emin"]
    Qs = {}
    for i in np.flatnonzero(~coarse):
        a, b = rp[i], rp[i + 1]
        m = b - a
        if m == 0:
            continue
        B = TV[c2glo[ci[a:b]], :]
        g = TV[i, :] - B.T @ p0[a:b]
        done = False
        if m > ntv:
            Q, R = np.linalg.qr(B, mode="reduced")
            d = np.abs(np.diag(R))
            if not d.max() / d.min() > condmax:
                y = scipy.linalg.solve_triangular(R, g, trans="T", lower=False)
                p0[a:b] += Q @ y
                Qs[i] = Q
                done = True
        if not done:
            U, sv, Vt = np.linalg.svd(B, full_matrices=False)
            r = 0
            if sv[0] > 1e-15:
                r = 1
                if m > 1:
                    while sv[0] < condmax * abs(sv[r]):
                        r += 1
                        if r == min(ntv, m):
                            break
            if r > 0:
                w = (Vt[:r, :] @ g) / sv[:r]
                p0[a:b] += U[:, :r] @ w
            Q = np.zeros((m, ntv))
            Q[:, :r] = U[:, :r]
            Qs[i] = Q

    def orth(x):
        y = x.copy()
        for i, Q in Qs.items():
            a, b = rp[i], rp[i + 1]
            y[a:b] = _orth_q(Q, b - a, x[a:b])
        return y

    # gather_f (A symmetric: A(c, i) = A(i, c))
    Ad = A.toarray() if n <= 20000 else None
    if Ad is not None:
        f = -Ad[c2glo[ci], rows] if nt else np.zeros(0)
    else:
        f = -np.asarray(A[c2glo[ci], rows]).ravel()
    dA = A.diagonal()
    tr_a = float(dA[coarse].sum())
    dinv = np.where(np.abs(dA) > 1e-15, 1.0 / np.where(dA == 0, 1.0, dA), 1.0)[rows]

    def kp(x):
        X = sp.csr_matrix((x, ci, rp), shape=(n, nc))
        C = (A @ X).tocsr()
        return np.asarray(C[rows, ci]).ravel() if nt else np.zeros(0)

    v = kp(p0)
    init_energy = tr_a + p0 @ v - 2.0 * (p0 @ f)
    res = orth(v - f)
    dp = np.zeros(nt)
    it = 0
    itmax, en_tol = prm["itmax_emin"], prm["energ_tol"]
    exit_test = itmax <= 0 or np.linalg.norm(res) < 1e-15
    gamma_old, pvec, de0 = 0.0, None, 1.0
    while not exit_test:
        it += 1
        z = orth(dinv * res)
        gamma = res @ z
        pvec = z.copy() if it == 1 else z + (gamma / gamma_old) * pvec
        gamma_old = gamma
        qkp = orth(kp(pvec))
        denom = qkp @ pvec
        if abs(denom) < 1e-18:
            break
        dek = gamma * gamma / denom
        alpha = gamma / denom
        dp += alpha * pvec
        res -= alpha * qkp
        if it == 1:
            de0 = dek
        exit_test = it == itmax or dek / de0 < en_tol
    del init_energy
    pf = p0 - dp
    # Prol_add_Cnodes + sparse(): coarse rows -> identity, exact zeros dropped
    r_out = np.concatenate([rows, c2glo])
    c_out = np.concatenate([ci, np.arange(nc)])
    v_out = np.concatenate([pf, np.ones(nc)])
    Pout = sp.csr_matrix((v_out, (r_out, c_out)), shape=(n, nc))
    Pout.eliminate_zeros()
    Pout.sort_indices()
    return Pout, it


def lmax_eigs(A, tol=1e-3, maxiter=3):
    """eigs(A,1,'lm',...) used by computeAMG.m:6 for the Dirichlet fix."""
    v0 = np.ones(A.shape[0]) / np.sqrt(A.shape[0])
    try:
        lam = spla.eigsh(A, k=1, which="LM", tol=tol, v0=v0, return_eigenvectors=False,
                         maxiter=max(maxiter * A.shape[0], 1000))
    except spla.ArpackNoConvergence as e:
        lam = e.eigenvalues
    return float(abs(lam[0]))


def diag_fix(A):
    """computeAMG.m:5-10: diagonal entries equal to 1 become lambda_max/10."""
    A = sp.csr_matrix(A, copy=True)
    d = A.diagonal()
    idx = d == 1
    if np.any(idx):
        lmax = lmax_eigs(A)
        d[idx] = lmax / 10.0
        A.setdiag(d)
    return A


# ----------------------------------------------------------------------------
# Synthetic problem generators (the reference ships none; these stand in for
# the configurations the path is measured on)
# ----------------------------------------------------------------------------

def poisson3d(nx, ny=None, nz=None):
    """7-point FD Laplacian on nx*ny*nz interior unknowns, Dirichlet boundary
    eliminated (no identity rows)."""
    ny = ny or nx
    nz = nz or nx
    def lap1(m):
        return sp.diags([-np.ones(m - 1), 2 * np.ones(m), -np.ones(m - 1)], [-1, 0, 1])
    Ix, Iy, Iz = sp.identity(nx), sp.identity(ny), sp.identity(nz)
    A = (sp.kron(Iz, sp.kron(Iy, lap1(nx))) + sp.kron(Iz, sp.kron(lap1(ny), Ix))
         + sp.kron(lap1(nz), sp.kron(Iy, Ix))).tocsr()
    A.sort_indices()
    return A


def mk_rbm_3d(X):
    """mk_rbm_3d.m:1-27: six rigid-body modes of 3-DOF nodes at coordinates X."""
    nn = X.shape[0]
    R = np.zeros((3 * nn, 6))
    R[0::3, 0] = 1
    R[1::3, 1] = 1
    R[2::3, 2] = 1
    XB = X.sum(axis=0) / nn
    R[1::3, 3] = -X[:, 2] + XB[2]
    R[2::3, 3] = X[:, 1] - XB[1]
    R[0::3, 4] = X[:, 2] - XB[2]
    R[2::3, 4] = -X[:, 0] + XB[0]
    R[0::3, 5] = -X[:, 1] + XB[1]
    R[1::3, 5] = X[:, 0] - XB[0]
    return R
