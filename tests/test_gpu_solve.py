"""GPU hierarchy, V-cycle and Krylov parity against the oracle, through the C ABI."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg  # noqa: F401

from conftest import rowwise_close
import chronoslab_b200 as cb
from chronoslab_b200 import problems as PB
from oracle import amg_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def oracle_from_gpu(h):
    """Oracle hierarchy built from the GPU hierarchy's own level matrices."""
    parts = []
    for l in range(h.nlevels):
        info = h.level_info(l)
        p = {"A": h.export(l, "A")}
        if l < h.nlevels - 1:
            p.update(G=h.export(l, "G"), P=h.export(l, "P"), omega=info["omega"])
        parts.append(p)
    return O.hierarchy_from_parts(parts)


@pytest.fixture(scope="module")
def elast():
    A, X = PB.elasticity_q1(10, return_coords=True)
    return A, PB.rbm_test_space(X), PB.elasticity_rhs(A, X, seed=0)


@pytest.fixture(scope="module")
def poisson():
    A = PB.poisson7(20)
    return A, np.ones((A.shape[0], 1)), PB.uniform_rhs(A.shape[0], seed=1)


@pytest.mark.parametrize("prec,tol", [(cb.CHRONOS_FP64, 1e-12), (cb.CHRONOS_FP32, 2e-5)])
@pytest.mark.parametrize("case", ["elast", "poisson"])
def test_vcycle_parity(lib, case, prec, tol, request):
    A, TV, b = request.getfixturevalue(case)
    ntv = TV.shape[1]
    with cb.Hierarchy(A, TV, cb.params(precision=prec, ntv=ntv)) as h:
        assert h.nlevels >= 2
        Ho = oracle_from_gpu(h)
        x = h.vcycle(b)
        xo = O.amg_vcycle(Ho, b)
        assert rel(x, xo) <= tol


@pytest.mark.parametrize("case", ["elast", "poisson"])
def test_pcg_iterations_fp64(lib, case, request):
    A, TV, b = request.getfixturevalue(case)
    ntv = TV.shape[1]
    with cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP64, ntv=ntv)) as h:
        Ho = oracle_from_gpu(h)
        x, it, rv, flag, _ = h.pcg(b, itmax=500, tol=1e-8)
        xo, ito, rvo, flago = O.pcg_cj(lambda r: O.amg_vcycle(Ho, r), lambda v: A @ v, b,
                                       np.zeros_like(b), 500, 1e-8)
        assert flag == 0 and flago == 0
        assert abs(it - ito) <= 1
        assert rv.shape == (it + 1,)
        assert np.allclose(rv[:min(it, ito)], rvo[:min(it, ito)], rtol=1e-6, atol=0)
        assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) <= 1e-8


@pytest.mark.parametrize("case", ["elast", "poisson"])
def test_pcg_fp32_hierarchy(lib, case, request):
    """FP32 hierarchy + FP64 outer PCG reaches the FP64 true residual and agrees
    with the FP64 oracle solve."""
    A, TV, b = request.getfixturevalue(case)
    ntv = TV.shape[1]
    with cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP32, ntv=ntv)) as h32, \
            cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP64, ntv=ntv)) as h64:
        x32, it32, _, f32, _ = h32.pcg(b, itmax=500, tol=1e-8)
        x64, it64, _, f64, _ = h64.pcg(b, itmax=500, tol=1e-8)
        assert f32 == 0 and f64 == 0
        assert np.linalg.norm(b - A @ x32) / np.linalg.norm(b) <= 1e-8
        assert abs(it32 - it64) <= 2
        xs = sp.linalg.spsolve(A.tocsc(), b)
        assert rel(x32, xs) <= 1e-6


@pytest.mark.parametrize("prec,tol", [(cb.CHRONOS_FP64, 1e-12), (cb.CHRONOS_FP32, 2e-5)])
def test_block_form_matches_csr(lib, elast, prec, tol):
    """The 3x3 block form of the level-1 operator gives the CSR results."""
    A, TV, b = elast
    with cb.Hierarchy(A, TV, cb.params(precision=prec, use_bsr=1)) as hb, \
            cb.Hierarchy(A, TV, cb.params(precision=prec, use_bsr=0)) as hc:
        assert hb.level_info(0)["block_rows"] == A.shape[0] // 3
        assert hc.level_info(0)["block_rows"] == 0
        assert rel(hb.vcycle(b), hc.vcycle(b)) <= tol
        xb, itb, _, fb, _ = hb.pcg(b, itmax=500, tol=1e-8)
        xc, itc, _, fc, _ = hc.pcg(b, itmax=500, tol=1e-8)
        assert fb == 0 and fc == 0 and abs(itb - itc) <= 1
        assert np.linalg.norm(b - A @ xb) / np.linalg.norm(b) <= 1e-8


def test_block_form_not_used_without_blocks(lib, poisson):
    A, _, b = poisson
    with cb.Hierarchy(A, np.ones(A.shape[0]), cb.params(ntv=1)) as h:
        assert h.level_info(0)["block_rows"] == 0


def test_graph_loop_matches_host_loop(lib, elast):
    A, TV, b = elast
    out = []
    for g in (1, 0):
        with cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP32, use_graph=g)) as h:
            x, it, rv, flag, _ = h.pcg(b, itmax=500, tol=1e-8)
            out.append((x, it, rv))
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])          # deterministic reductions


def test_pcg_repeatable_and_x0(lib, poisson):
    A, _, b = poisson
    with cb.Hierarchy(A, np.ones(A.shape[0]), cb.params(ntv=1)) as h:
        x1, it1, _, _, _ = h.pcg(b, itmax=500, tol=1e-8)
        x2, it2, _, _, _ = h.pcg(b, itmax=500, tol=1e-8)
        assert it1 == it2 and np.array_equal(x1, x2)
        # warm start at the solution: PCG_CJ always takes one iteration
        x3, it3, rv3, flag3, _ = h.pcg(b, x0=x1, itmax=500, tol=1e-8)
        assert it3 == 1 and flag3 == 0
        # zero right-hand side returns zero, no iterations (PCG_CJ.m:12-16)
        x4, it4, _, flag4, _ = h.pcg(np.zeros_like(b), itmax=500, tol=1e-8)
        assert it4 == 0 and flag4 == 0 and not np.any(x4)
        # itmax reached -> flag 1 (PCG_CJ.m:69-71)
        _, it5, _, flag5, _ = h.pcg(b, itmax=2, tol=1e-14)
        assert it5 == 2 and flag5 == 1


def test_cubo_end_to_end_pinned(lib, cubo, cubo_ref):
    """The reference's pinned regression: SQMR to 1e-6 on Cubo_4820 with the
    Tests/parm_* settings takes 43 iterations, tolerance max(5%, 2)
    (Tests/CubeBAMG_NONE.m:3,34)."""
    A, Af, TV0 = cubo["A"], cubo["Af"], cubo["TV0"]
    ref_it = cubo_ref["info"]["reference_sqmr_iterations"]
    with cb.Hierarchy(Af, TV0, cb.params(precision=cb.CHRONOS_FP64)) as h:
        assert h.level_info(0)["nnz_G"] == cubo_ref["info"]["nnz_G_level1"]
        assert h.level_info(0)["nc"] == cubo_ref["info"]["nc_level1"]
        # SQMR's operator is the unmodified A, the preconditioner uses Af
        x, info, relres, niter = h.sqmr(np.ones(A.shape[0]), 1e-6, 100, A=A)
        assert info == 0
        assert abs(niter - cubo_ref["info"]["oracle_sqmr_iterations"]) <= 1
        assert not (abs(ref_it / niter - 1) > 0.05 and abs(ref_it - niter) > 2)
        x, it, _, flag, _ = h.pcg(np.ones(A.shape[0]), itmax=200, tol=1e-8)
        assert flag == 0
        assert abs(it - cubo_ref["info"]["oracle_pcg_iterations_1e-8"]) <= 1


def test_cubo_smoothed_prolongation_pinned(lib, cubo, cubo_ref):
    """Jacobi-smoothed prolongation (prol_emin = SMOOTH): the reference's
    pinned regression takes 29 SQMR iterations to 1e-6 on Cubo_4820,
    tolerance max(5%, 2) (Tests/CubeBAMG_SMOOTH.m:3); the oracle restatement
    with the reference's BAMG C++ takes the golden count (within 1)."""
    A, Af, TV0 = cubo["A"], cubo["Af"], cubo["TV0"]
    info = cubo_ref["info"]
    ref_it = info["reference_sqmr_iterations_smooth"]
    with cb.Hierarchy(Af, TV0, cb.params(precision=cb.CHRONOS_FP64, prol_emin="SMOOTH")) as h:
        assert [h.level_info(l)["n"] for l in range(h.nlevels)] == info["levels_smooth"]
        P = h.export(0, "P")
        Ac = h.export(1, "A")
        assert rel(Ac.toarray(), (P.T @ (Af @ P)).toarray()) <= 1e-13
        x, sinfo, relres, niter = h.sqmr(np.ones(A.shape[0]), 1e-6, 100, A=A)
        assert sinfo == 0
        assert abs(niter - info["oracle_sqmr_iterations_smooth"]) <= 1
        assert not (abs(ref_it / niter - 1) > 0.05 and abs(ref_it - niter) > 2)
        x, it, _, flag, _ = h.pcg(np.ones(A.shape[0]), itmax=200, tol=1e-8)
        assert flag == 0
        assert abs(it - info["oracle_pcg_iterations_1e-8_smooth"]) <= 1
    # the smoothed operator P has wider rows than BAMG's
    assert P.nnz > cubo_ref["P"].nnz


def test_setup_components_match_golden(lib, cubo, cubo_ref):
    with cb.Hierarchy(cubo["Af"], cubo["TV0"], cb.params(precision=cb.CHRONOS_FP64)) as h:
        G = h.export(0, "G")
        Gref = cubo_ref["G"]
        assert np.array_equal(G.indptr, Gref.indptr) and np.array_equal(G.indices, Gref.indices)
        assert rowwise_close(G, Gref, 1e-10)
        P = h.export(0, "P")
        D = (P - cubo_ref["P"]).tocsr()
        bad_rows = np.unique(D.nonzero()[0][np.abs(D.data) > 1e-10])
        # The hierarchy orthonormalises TV twice (cpt_aspAMG.m:46 and tspace
        # NONE), our Householder QR rounding differs from LAPACK's, and the
        # Cubo rigid-body test space puts many BAMG rows on a knife edge (row
        # norm at maxrownrm, maxVol ties): a few rows pick another, equally
        # exact, interpolation set.  Same inputs: test_host's BAMG check.
        assert bad_rows.size <= 0.01 * P.shape[0]
        TVc = cubo["TV0"][np.flatnonzero(cubo_ref["fcnode"] > 0)]
        ok = cubo_ref["c_mark"] == 0
        err = np.linalg.norm(P @ TVc - cubo["TV0"], axis=1)
        assert np.all(err[ok] <= 1e-8 * np.linalg.norm(cubo["TV0"], axis=1)[ok] + 1e-14)
        # the coarse operator is the Galerkin product of the exported P
        Ac = h.export(1, "A")
        ref = (P.T @ (cubo["Af"] @ P)).tocsr()
        assert rel(Ac.toarray(), ref.toarray()) <= 1e-13
        info = h.level_info(0)
        assert 0.0 < info["omega"] <= 1.0


@pytest.mark.parametrize("ratio", [0.01, 0.5])
@pytest.mark.parametrize("case", ["elast", "poisson"])
def test_outer_fp32_values_with_replacement(lib, case, ratio, request):
    """FP32 hierarchy, outer A p from the stored FP32 level-1 values with FP64
    accumulation and FP64 true-residual replacement (the default) against the
    FP64 outer operator on the same hierarchy: iterations within 1, the true
    residual below the tolerance, the same solution, and the last residual
    reported is the true one."""
    A, TV, b = request.getfixturevalue(case)
    ntv = TV.shape[1]
    with cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP32, ntv=ntv,
                                       replace_ratio=ratio)) as hm, \
            cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP32, ntv=ntv,
                                          exact_outer=1)) as he:
        xm, itm, rvm, fm, _ = hm.pcg(b, itmax=500, tol=1e-8)
        xe, ite, rve, fe, _ = he.pcg(b, itmax=500, tol=1e-8)
        assert fm == 0 and fe == 0
        assert abs(itm - ite) <= 1
        true_m = np.linalg.norm(b - A @ xm) / np.linalg.norm(b)
        assert true_m <= 1e-8
        assert rvm[-1] == pytest.approx(true_m, rel=1e-6)
        assert rel(xm, xe) <= 1e-7


def test_outer_replacement_itmax_and_warm_start(lib, elast):
    A, TV, b = elast
    with cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP32)) as h:
        # itmax reached: flag 1, the final residual is the true one
        x, it, rv, flag, _ = h.pcg(b, itmax=3, tol=1e-14)
        assert it == 3 and flag == 1
        true = np.linalg.norm(b - A @ x) / np.linalg.norm(b)
        assert rv[-1] == pytest.approx(true, rel=1e-6)
        # warm start at the solution: one iteration
        xs, _, _, _, _ = h.pcg(b, itmax=500, tol=1e-8)
        x3, it3, _, flag3, _ = h.pcg(b, x0=xs, itmax=500, tol=1e-8)
        assert it3 == 1 and flag3 == 0


@pytest.mark.parametrize("prec,tol", [(cb.CHRONOS_FP64, 1e-12), (cb.CHRONOS_FP32, 2e-5)])
@pytest.mark.parametrize("case", ["elast", "poisson"])
def test_sliced_ell_matches_csr(lib, case, prec, tol, request):
    """The sliced ELL form of the short-row operators (G, G', P and the
    7-point A) gives the row-grouped CSR results."""
    A, TV, b = request.getfixturevalue(case)
    ntv = TV.shape[1]
    with cb.Hierarchy(A, TV, cb.params(precision=prec, ntv=ntv, spmv_format=2)) as he, \
            cb.Hierarchy(A, TV, cb.params(precision=prec, ntv=ntv, spmv_format=1)) as hc:
        assert he.level_info(0)["sell_mask"] & 0b01110       # G, G', P at level 1
        assert hc.level_info(0)["sell_mask"] == 0
        if case == "poisson":
            assert he.level_info(0)["sell_mask"] & 1         # the 7-point operator itself
        assert rel(he.vcycle(b), hc.vcycle(b)) <= tol
        xe, ite, _, fe, _ = he.pcg(b, itmax=500, tol=1e-8)
        xc, itc, _, fc, _ = hc.pcg(b, itmax=500, tol=1e-8)
        assert fe == 0 and fc == 0 and abs(ite - itc) <= 1
        assert np.linalg.norm(b - A @ xe) / np.linalg.norm(b) <= 1e-8


def test_plain_stream_order_matches_pdl(lib, elast, tmp_path):
    """CHRONOS_PDL=0 (plain stream order instead of programmatic dependent
    launch; read once per process, so in a child process) gives the same
    solution bit for bit."""
    import os
    import subprocess
    import sys
    A, TV, b = elast
    with cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP32)) as h:
        x, it, _, flag, _ = h.pcg(b, itmax=500, tol=1e-8)
    inp = tmp_path / "case.npz"
    out = tmp_path / "x.npy"
    np.savez(inp, data=A.data, indices=A.indices, indptr=A.indptr, TV=TV, b=b)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = (
        "import sys, numpy as np, scipy.sparse as sp\n"
        f"sys.path.insert(0, {root!r})\n"
        "import chronoslab_b200 as cb\n"
        f"z = np.load({str(inp)!r})\n"
        "A = sp.csr_matrix((z['data'], z['indices'], z['indptr']))\n"
        "with cb.Hierarchy(A, z['TV'], cb.params(precision=cb.CHRONOS_FP32)) as h:\n"
        "    x, it, _, flag, _ = h.pcg(z['b'], itmax=500, tol=1e-8)\n"
        f"np.save({str(out)!r}, np.append(x, [it, flag]))\n")
    env = dict(os.environ, CHRONOS_PDL="0")
    subprocess.run([sys.executable, "-c", code], env=env, check=True, timeout=600)
    y = np.load(out)
    assert int(y[-2]) == it and int(y[-1]) == flag == 0
    assert np.array_equal(y[:-2], x)


def test_hierarchy_dump_ext_bin(lib, elast, tmp_path):
    """A level operator written by the hierarchy in .Ext_bin reads back as the
    exported operator (FP64 values)."""
    A, TV, b = elast
    with cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP32)) as h:
        for lvl, which in ((0, "A"), (0, "P"), (1, "A")):
            p = tmp_path / f"L{lvl}{which}.Ext_bin"
            h.dump_ext_bin(lvl, which, str(p))
            E = h.export(lvl, which)
            R = cb.read_ext_bin(str(p))
            R = R[:, :E.shape[1]] if which == "P" else R
            assert R.shape[0] == E.shape[0] and (R != E).nnz == 0


@pytest.mark.parametrize("prec", [cb.CHRONOS_FP32, cb.CHRONOS_FP64])
def test_hierarchy_save_load_round_trip(lib, elast, tmp_path, prec):
    """A hierarchy written to a file and read back without the setup has the
    same levels, operators and omegas, and gives the same V-cycle and PCG
    solve bit for bit."""
    A, TV, b = elast
    path = str(tmp_path / "elast.chh")
    with cb.Hierarchy(A, TV, cb.params(precision=prec)) as h:
        h.save(path)
        info = [h.level_info(l) for l in range(h.nlevels)]
        z = h.vcycle(b)
        x, it, rv, flag, _ = h.pcg(b, itmax=500, tol=1e-8)
        ops = [(h.export(l, "A"), h.export(l, "G") if l < h.nlevels - 1 else None)
               for l in range(h.nlevels)]
    with cb.Hierarchy.load(path) as g:
        assert g.nlevels == len(info) and g.n == A.shape[0]
        for l, i in enumerate(info):
            j = g.level_info(l)
            assert (j["n"], j["nnz_A"], j["nnz_G"], j["nnz_P"], j["nc"]) == \
                (i["n"], i["nnz_A"], i["nnz_G"], i["nnz_P"], i["nc"])
            assert j["omega"] == i["omega"]
            Al, Gl = ops[l]
            assert (g.export(l, "A") != Al).nnz == 0
            if Gl is not None:
                assert (g.export(l, "G") != Gl).nnz == 0
        assert np.array_equal(g.vcycle(b), z)
        y, it2, rv2, flag2, _ = g.pcg(b, itmax=500, tol=1e-8)
    assert it2 == it and flag2 == flag == 0
    assert np.array_equal(y, x) and np.array_equal(rv2, rv)


def test_amg_info_complexities(lib, elast):
    """get_AMG_info's statistics from the exported level matrices: grid and
    operator complexity, coarse sizes and prolongation entries."""
    A, TV, b = elast
    with cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP32)) as h:
        info = h.amg_info()
        mats = [h.export(l, "A") for l in range(h.nlevels)]
        Ps = [h.export(l, "P") for l in range(h.nlevels - 1)]
    assert len(info) == len(mats) >= 2
    assert info[0]["grid_comp"] == pytest.approx(sum(M.shape[0] for M in mats) / mats[0].shape[0])
    assert info[0]["oper_comp"] == pytest.approx(sum(M.nnz for M in mats) / mats[0].nnz)
    for l, P in enumerate(Ps):
        assert info[l]["nc"] == P.shape[1] == mats[l + 1].shape[0]
        assert info[l]["nt_P"] == P.nnz
    n_c = mats[-1].shape[0]
    assert info[-1]["nt_L"] == n_c * (n_c + 1) // 2


def test_c1_poisson32_against_the_reference_hierarchy(lib):
    """The C1 configuration at full size (7-point Poisson 32^3, RHS U[-1,1],
    x0 = 0, PCG_CJ to 1e-8): the GPU solve (FP64 and FP32 hierarchies) takes
    the iteration count of the CPU path built with the reference's own FSAI
    and BAMG C++ (oracle/_ref) within one, and agrees with its solution."""
    from oracle import c_oracle as CO
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    A = PB.poisson7(32)
    n = A.shape[0]
    b = PB.uniform_rhs(n, seed=0)
    prm = O.default_params()
    prm["tspace"]["ntv"] = 1
    CH = CO.CHierarchy(CO.reference_hierarchy(A, np.ones((n, 1)), prm))
    xo, ito, _, flo = CH.pcg(b, itmax=500, tol=1e-8)
    assert flo == 0
    for prec in (cb.CHRONOS_FP64, cb.CHRONOS_FP32):
        with cb.Hierarchy(A, np.ones((n, 1)), cb.params(precision=prec, ntv=1)) as h:
            x, it, _, flag, _ = h.pcg(b, itmax=500, tol=1e-8)
        assert flag == 0 and abs(it - ito) <= 1
        assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b)
        assert rel(x, xo) <= 1e-6


def test_elasticity_own_bamg_against_the_reference_hierarchy(lib):
    """Q1 elasticity 20^3 with the library's own coarsening and BAMG against
    the CPU path built with the reference's own FSAI and BAMG C++.  The first
    coarsening is the same (same operator and strength), so the first two
    level sizes agree.  Deeper down the BAMG interpolation sets differ in
    about a tenth of the rows: on a uniform grid the rigid-body test space
    makes many maximum-volume candidate sets tie, and the last bits of the
    test space's orthonormalisation (this library's Householder QR there,
    LAPACK's here) choose among them.  The iteration count of this path is
    therefore not held to the reference's (53 vs 50 measured); the
    within-one criterion is tested on the reference's own prolongation
    (test_gpu_reference_prolong.py).  Both solves reach the true relative
    residual 1e-8 and the same solution."""
    from oracle import c_oracle as CO
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    A, X = PB.elasticity_q1(20, return_coords=True)
    TV = PB.rbm_test_space(X)
    b = PB.elasticity_rhs(A, X, seed=0)
    H = CO.reference_hierarchy(A, TV, O.default_params())
    xo, ito, _, flo = CO.CHierarchy(H).pcg(b, itmax=500, tol=1e-8)
    assert flo == 0
    for prec in (cb.CHRONOS_FP64, cb.CHRONOS_FP32):
        with cb.Hierarchy(A, TV, cb.params(precision=prec)) as h:
            sizes = [h.level_info(l)["n"] for l in range(h.nlevels)]
            ref = [lv.A.shape[0] for lv in H.levels]
            assert len(sizes) == len(ref) and sizes[:2] == ref[:2]
            x, it, _, flag, _ = h.pcg(b, itmax=500, tol=1e-8)
        assert flag == 0
        assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b)
        assert rel(x, xo) <= 1e-6


def test_lambda_and_omega_against_eigs(lib, cubo):
    """smoother.m:73-81: lambda_max(F A F') by eigs(...,'la', tol 5e-4) and
    omega = min(1, 1.9/lambda).  The GPU Lanczos value on every smoothing
    level of Cubo agrees with ARPACK's (scipy eigsh, same tolerance) on the
    GPU's own level operator and factor within 5e-4 relative; so does omega."""
    with cb.Hierarchy(cubo["Af"], cubo["TV0"], cb.params(precision=cb.CHRONOS_FP64)) as h:
        assert h.nlevels >= 2
        for l in range(h.nlevels - 1):
            info = h.level_info(l)
            lam = O.lambda_max_fsai(h.export(l, "A"), h.export(l, "G"))
            assert abs(info["lambda"] - lam) <= 5e-4 * lam, (l, info["lambda"], lam)
            om = min(1.0, 1.9 / lam)
            assert abs(info["omega"] - om) <= 5e-4 * om


def test_diag_fix_against_eigs(lib, cubo):
    """computeAMG.m:5-10: diagonal entries equal to 1 (Cubo's Dirichlet rows)
    become lambda_max(A)/10, eigs tolerance 1e-3; every other entry is kept."""
    A = cubo["A"]
    d = A.diagonal()
    idx = np.flatnonzero(d == 1.0)
    assert idx.size > 0
    Ag = cb.diag_fix(A)
    Ao = O.diag_fix(A)
    dg, do = Ag.diagonal(), Ao.diagonal()
    assert np.all(np.abs(dg[idx] - do[idx]) <= 1e-3 * do[idx])
    keep = np.setdiff1d(np.arange(A.shape[0]), idx)
    assert np.array_equal(dg[keep], d[keep])
    off = (Ag - sp.diags(dg)) - (A - sp.diags(d))
    assert abs(off).max() == 0.0


def test_setup_phases_sum_to_total(lib, elast):
    """Every second of the setup falls in a named phase: the twelve entries
    minus the total sum to the total, and the named ones are not negative."""
    A, TV, b = elast
    with cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP32)) as h:
        t = h.setup_times()
    assert len(t) == 12 and all(v >= 0.0 for v in t.values())
    parts = sum(v for k, v in t.items() if k != "total")
    assert abs(parts - t["total"]) <= 1e-6 * max(t["total"], 1.0) + 1e-9
    assert t["uploads"] > 0.0 and t["layouts"] > 0.0
