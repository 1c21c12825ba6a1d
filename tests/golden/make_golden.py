"""Generates the golden fixtures of the parity tests from the reference itself.

Run here, where the reference is mounted (it does not exist on the GPU
machine, so the fixtures are committed):

    make -C oracle ref && python tests/golden/make_golden.py [REFERENCE_ROOT]

Writes, next to this script:
  cubo_A_upper.npz   Cubo_4820 (examples/matrices/Cubo_4820.mat): upper
                     triangle of A (symmetric), TV0, and the diagonal value
                     lambda_max/10 that computeAMG.m:5-10 writes into the
                     unit-diagonal (Dirichlet) rows, computed once here so
                     every test uses the same matrix.
  cubo_ref_fsai.npz  the reference's compute_local_fsai (oracle/_ref, built
                     from MEX_SYM_AFSAI unmodified) on that matrix with the
                     Tests/parm_SMOOTH settings 15 / 1 / 1e-3.
  cubo_ref_bamg.npz  the reference's BAMG (oracle/_ref) on the oracle's C/F
                     splitting of that matrix (DOM 0.01, PMIS, rng(0)) with
                     TV = qr(TV0) and Tests/parm_PROLONG settings.
  small_ref.npz      the reference FSAI on small Poisson (8^3) and Q1
                     elasticity (4^3 elements) matrices.
  cubo_ref.json      reference-pinned and oracle iteration counts (also with
                     the Jacobi-smoothed and the energy-minimised
                     prolongations; the EMIN keys come from emin_counts,
                     which can be rerun alone: make_golden.py --emin).
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import amg_oracle as O            # noqa: E402
from chronoslab_b200 import problems as PB   # noqa: E402


def save_csr(path, **mats_and_arrays):
    out = {}
    for k, v in mats_and_arrays.items():
        if sp.issparse(v):
            v = sp.csr_matrix(v)
            out[k + "_indptr"] = v.indptr.astype(np.int64)
            out[k + "_indices"] = v.indices.astype(np.int32)
            out[k + "_data"] = v.data.astype(np.float64)
            out[k + "_shape"] = np.array(v.shape, dtype=np.int64)
        else:
            out[k] = np.asarray(v)
    np.savez_compressed(path, **out)


def main(ref_root):
    mat = os.path.join(ref_root, "examples", "matrices", "Cubo_4820.mat")
    m = O.load_mat(mat)
    A = m["A"].tocsr()
    A.sort_indices()
    TV0 = m["TV0"]
    lmax = O.lmax_eigs(A)
    fixval = lmax / 10.0
    U = sp.triu(A).tocsr()
    np.savez_compressed(os.path.join(HERE, "cubo_A_upper.npz"),
                        indptr=U.indptr.astype(np.int32), indices=U.indices.astype(np.int32),
                        data=U.data, n=np.int64(A.shape[0]), TV0=TV0, diag_fix=np.float64(fixval))
    Af = A.copy()
    d = Af.diagonal()
    d[d == 1.0] = fixval
    Af.setdiag(d)
    Af.sort_indices()

    prm = O.default_params(8)
    G, posdef = O.ref_afsai(Af, 8, 15, 1, 1e-3)
    save_csr(os.path.join(HERE, "cubo_ref_fsai.npz"), G=G, posdef=np.int64(posdef))

    rng = O.MatlabRand()
    fc, clist, flist, S = O.coarsen(prm["coarsen"], Af, rng)
    TV = O.qr_thin(TV0)
    P, cmark = O.ref_bamg(prm["prolong"], clist.size, fc, S, TV)
    save_csr(os.path.join(HERE, "cubo_ref_bamg.npz"), P=P, fcnode=fc.astype(np.int32),
             c_mark=cmark.astype(np.int8), nc=np.int64(clist.size), S_nnz=np.int64(S.nnz))

    # small matrices
    Ap = PB.poisson7(8)
    Ae, _ = PB.elasticity_q1(4, return_coords=True)
    Gp, _ = O.ref_afsai(Ap, 2, 15, 1, 1e-3)
    Ge, _ = O.ref_afsai(Ae, 2, 15, 1, 1e-3)
    save_csr(os.path.join(HERE, "small_ref.npz"), Ap=Ap, Gp=Gp, Ae=Ae, Ge=Ge)

    # end-to-end oracle runs with the reference's own C++ kernels
    H = O.cpt_aspamg(prm, Af, TV0)
    Mv = lambda r: O.amg_vcycle(H, r, 0, Af)
    rhs = np.ones(A.shape[0])
    _, info, relres, niter, _ = O.sqmr(lambda v: A @ v, rhs, 1e-6, 100, Mv)
    _, it, _, flag = O.pcg_cj(Mv, lambda v: Af @ v, rhs, np.zeros_like(rhs), 1000, 1e-8)
    # Jacobi-smoothed prolongation (prolong.m:180-196), Tests/CubeBAMG_SMOOTH.m
    prm_s = O.default_params(8)
    prm_s["prolong"]["prol_emin"] = "SMOOTH"
    Hs = O.cpt_aspamg(prm_s, Af, TV0)
    Mvs = lambda r: O.amg_vcycle(Hs, r, 0, Af)
    _, info_s, relres_s, niter_s, _ = O.sqmr(lambda v: A @ v, rhs, 1e-6, 100, Mvs)
    _, it_s, _, _ = O.pcg_cj(Mvs, lambda v: Af @ v, rhs, np.zeros_like(rhs), 1000, 1e-8)
    info_out = emin_counts(A, Af, TV0)
    info_out.update({
        "reference_sqmr_iterations_smooth": 29,
        "reference_sqmr_source_smooth": "Tests/CubeBAMG_SMOOTH.m:3 (tolerance max(5%, 2))",
        "oracle_sqmr_iterations_smooth": int(niter_s),
        "oracle_pcg_iterations_1e-8_smooth": int(it_s),
        "levels_smooth": [int(L.A.shape[0]) for L in Hs.levels],
        "reference_sqmr_iterations": 43,
        "reference_sqmr_source": "Tests/CubeBAMG_NONE.m:3 (tolerance max(5%, 2), :34)",
        "oracle_sqmr_iterations": int(niter),
        "oracle_sqmr_relres": float(relres),
        "oracle_pcg_iterations_1e-8": int(it),
        "levels": [int(L.A.shape[0]) for L in H.levels],
        "nnz_G_level1": int(G.nnz),
        "nc_level1": int(clist.size),
        "diag_fix": float(fixval),
    })
    with open(os.path.join(HERE, "cubo_ref.json"), "w") as f:
        json.dump(info_out, f, indent=1)
    print(json.dumps(info_out, indent=1))


def emin_counts(A, Af, TV0):
    """Energy-minimised prolongation (prolong.m:207-235, the reference's EMIN
    C++ from oracle/_ref) on Cubo_4820, as Tests/CubeBAMG_EMIN.m runs it."""
    prm = O.default_params(8)
    prm["prolong"]["prol_emin"] = "EMIN"
    H = O.cpt_aspamg(prm, Af, TV0)
    Mv = lambda r: O.amg_vcycle(H, r, 0, Af)
    rhs = np.ones(A.shape[0])
    _, info, relres, niter, _ = O.sqmr(lambda v: A @ v, rhs, 1e-6, 100, Mv)
    _, it, _, _ = O.pcg_cj(Mv, lambda v: Af @ v, rhs, np.zeros_like(rhs), 1000, 1e-8)
    return {
        "reference_sqmr_iterations_emin": 20,
        "reference_sqmr_source_emin": "Tests/CubeBAMG_EMIN.m:3 (tolerance max(5%, 2), :34)",
        "oracle_sqmr_iterations_emin": int(niter),
        "oracle_pcg_iterations_1e-8_emin": int(it),
        "levels_emin": [int(L.A.shape[0]) for L in H.levels],
    }


def update_emin_counts():
    """Adds the EMIN keys to an existing cubo_ref.json (the other fixtures
    are left as they are)."""
    z = np.load(os.path.join(HERE, "cubo_A_upper.npz"))
    n = int(z["n"])
    U = sp.csr_matrix((z["data"], z["indices"], z["indptr"]), shape=(n, n))
    A = (U + sp.triu(U, 1).T).tocsr()
    A.sort_indices()
    Af = A.copy()
    d = Af.diagonal()
    d[d == 1.0] = float(z["diag_fix"])
    Af.setdiag(d)
    Af.sort_indices()
    path = os.path.join(HERE, "cubo_ref.json")
    with open(path) as f:
        info = json.load(f)
    info.update(emin_counts(A, Af, z["TV0"]))
    with open(path, "w") as f:
        json.dump(info, f, indent=1)
    print(json.dumps(info, indent=1))


if __name__ == "__main__":
    if sys.argv[1:] == ["--emin"]:
        update_emin_counts()
        sys.exit(0)
    from oracle.refdir import reference_dir
    ref = sys.argv[1] if len(sys.argv) > 1 else reference_dir()
    if not ref:
        sys.exit("reference tree not found: pass its path or set CHRONOS_REFERENCE_DIR")
    main(ref)
