"""Host-side setup restatements (no GPU) against the reference's own C++
(golden vectors made by oracle/_ref) and the oracle's MATLAB restatement."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import rowwise_close
import chronoslab_b200 as cb
from chronoslab_b200 import problems as PB
from oracle import amg_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_fsai_pattern_matches_reference_cubo(lib, cubo, cubo_ref):
    G, ok = cb.fsai_pattern(cubo["Af"], 15, 1, 1e-3, nthread=4)
    Gref = cubo_ref["G"]
    assert ok
    assert G.nnz == cubo_ref["info"]["nnz_G_level1"] == Gref.nnz
    assert np.array_equal(G.indptr, Gref.indptr) and np.array_equal(G.indices, Gref.indices)
    assert rowwise_close(G, Gref, 1e-10)


def test_fsai_pattern_small_reference(lib, small_ref):
    for A, Gref in ((small_ref["Ap"], small_ref["Gp"]), (small_ref["Ae"], small_ref["Ge"])):
        G, ok = cb.fsai_pattern(A, 15, 1, 1e-3)
        assert ok and np.array_equal(G.indices, Gref.indices) and np.array_equal(G.indptr, Gref.indptr)
        assert rowwise_close(G, Gref, 1e-10)


def test_fsai_pattern_properties(lib):
    """Rows list strictly-lower columns ascending then the diagonal; at most
    nstep*step_size off-diagonal entries; G A G' has unit diagonal."""
    A = PB.poisson7(6) * 10.0
    for nstep, step in ((15, 1), (5, 2), (0, 1)):
        G, ok = cb.fsai_pattern(A, nstep, step, 1e-3, fsai_fabs=1)
        assert ok
        for i in range(A.shape[0]):
            cols = G.indices[G.indptr[i]:G.indptr[i + 1]]
            assert cols[-1] == i and np.all(np.diff(cols[:-1]) > 0) and np.all(cols[:-1] < i)
            assert cols.size - 1 <= nstep * step
        M = (G @ A @ G.T).diagonal()
        assert np.allclose(M, 1.0, rtol=1e-12)


def test_fsai_reference_abs_truncation(lib):
    """The reference's int abs: with entries below 1 in magnitude the Kaporin
    decrease truncates to 0 and every row stops after two steps."""
    A = PB.poisson7(6) * 0.01
    G, _ = cb.fsai_pattern(A, 15, 1, 1e-3, fsai_fabs=0)
    assert np.max(np.diff(G.indptr)) <= 3
    G2, _ = cb.fsai_pattern(A, 15, 1, 1e-3, fsai_fabs=1)
    assert np.max(np.diff(G2.indptr)) > 3


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")
def test_fsai_pattern_vs_reference_library(lib):
    A = PB.elasticity_q1(5) * 1e4       # values above 1: the int abs keeps the ranking
    G, _ = cb.fsai_pattern(A, 15, 1, 1e-3, nthread=2)
    Gr, _ = O.ref_afsai(A, 2, 15, 1, 1e-3)
    assert np.array_equal(G.indptr, Gr.indptr) and np.array_equal(G.indices, Gr.indices)
    assert rowwise_close(G, Gr, 1e-10)


def test_coarsen_matches_oracle_and_golden(lib, cubo, cubo_ref):
    fc, nc, S = cb.coarsen(cubo["Af"], cb.params(), 0)
    assert nc == cubo_ref["nc"]
    assert np.array_equal(fc, cubo_ref["fcnode"])
    fco, clist, _, So = O.coarsen(O.default_params(2)["coarsen"], cubo["Af"], O.MatlabRand())
    assert np.array_equal(fc, fco)
    assert (S != So).nnz == 0


@pytest.mark.parametrize("soc,tau", [("DOM", 0.01), ("CLA", 0.25)])
def test_coarsen_small_matches_oracle(lib, soc, tau):
    A = PB.diffusion7(10, sigma=1.0, corr_len=3.0, seed=4)[0]
    for skip in (0, 37):
        fc, nc, S = cb.coarsen(A, cb.params(SoC_type=soc, soc_tau=tau), skip)
        rng = O.MatlabRand()
        if skip:
            rng.rand(skip)
        fco, clist, _, So = O.coarsen({"SoC_type": soc, "tau": tau}, A, rng)
        assert np.array_equal(fc, fco) and nc == clist.size
        assert abs(S - So).max() <= 1e-15


def test_mt19937_matches_matlab_rand(lib):
    """rng(0); rand -> 0.8147, 0.9058, 0.1270: PMIS weights of a graph without
    edges are exactly the random draws' order."""
    A = sp.identity(3, format="csr") * 2.0
    fc, nc, _ = cb.coarsen(A, cb.params(), 0)
    # Dirichlet-like columns (one nonzero) are all fine: nothing is drawn into a choice
    assert nc == 0
    r = O.MatlabRand().rand(3)
    assert np.allclose(r, [0.8147236863931789, 0.9057919370756192, 0.1269868162935061])


def test_bamg_matches_reference_golden(lib, cubo, cubo_ref):
    fc, nc, S = cb.coarsen(cubo["Af"], cb.params(), 0)
    TV = O.qr_thin(cubo["TV0"])
    P, cm = cb.bamg(S, fc, TV, cb.params(prol_np=4))
    Pref = cubo_ref["P"]
    D = (P - Pref).tocsr()
    bad_rows = np.unique(D.nonzero()[0][np.abs(D.data) > 1e-10])
    # identical up to rounding except where LAPACK rounding flips a knife-edge
    # test (a row norm exactly at maxrownrm): at most 0.1% of the rows
    assert bad_rows.size <= 0.001 * P.shape[0]
    assert cm.sum() == cubo_ref["c_mark"].sum()
    # exact interpolation of the test space on the F rows the reference fits exactly
    ok = cubo_ref["c_mark"] == 0
    TVc = TV[np.flatnonzero(fc > 0)]          # coarse nodes in coarse-index order
    err = np.linalg.norm(P @ TVc - TV, axis=1)
    assert np.all(err[ok] <= 1e-8 * np.maximum(np.linalg.norm(TV, axis=1)[ok], 1e-300) + 1e-14)


def test_params_files(lib, tmp_path):
    files = {
        "parm_AMG": "10   % nLevMax\n1000 % maxCoarseSZ\n",
        "parm_SMOOTH": "20 %\n1 %\n1 %\n15 %\n1 %\n1.e-3 %\nAFSAI_SYM %\n",
        "parm_TSPACE": "6 %\n40 %\n1.e-4 %\nNONE %\n5 %\n\nAvailable Methods:\n",
        "parm_COARSEN": "CLA %\n0.2 %\n0 %\n",
        "parm_PROLONG": "BAMG\nEMIN\n20\n100\n0.01\n1\n10\n1.e+13\n5.0\n1.e-10\n0\n3\n0.020\n25\n8\n"
                        "0.002\n1.e+9\n1\n3\n0\n20\n5\n",
        "parm_FILTER": "10\n170.0\n0.1\n0.000\n0\n",
        "parm_GENERAL": "false\nunit_rhs\ntrue\nPCG\n15000\n1.e-8\n100\n",
    }
    for k, v in files.items():
        (tmp_path / k).write_text(v)
    (tmp_path / "aspAMG.fnames").write_text("\n".join(files) + "\nThrash\nThrash\nThrash\nx.mat\n")
    p = cb.readDefaultParams(tmp_path / "aspAMG.fnames")
    assert p.SoC_type == b"CLA" and p.soc_tau == 0.2 and p.nthread == 20 and p.nstep == 15
    assert p.maxcond == 1e13 and p.itmax == 15000 and p.tol == 1e-8 and p.symmetric == 1
    assert p.tspace_method == b"NONE" and p.proltype == b"BAMG" and p.filt_wgt == 170.0
    # the EMIN lines of parm_PROLONG (read_prolong.m)
    assert p.prol_emin == b"EMIN" and p.patt_pow == 3 and p.patt_tau == 0.02
    assert p.nnzr_max == 25 and p.itmax_emin == 8 and p.energ_tol == 0.002
    assert p.condmax_emin == 1e9 and p.prec_emin == 1 and p.solv_emin == 3
    # the oracle reads the same files the same way
    q = O.read_params(str(tmp_path / "aspAMG.fnames"))
    assert q["coarsen"]["tau"] == p.soc_tau and q["smoother"]["nstep"] == p.nstep
    assert (q["prolong"]["patt_pow"], q["prolong"]["nnzr_max"], q["prolong"]["solv_emin"]) == (3, 25, 3)
    (tmp_path / "parm_AMG").write_text("10\n")
    with pytest.raises(cb.ChronosError) as e:
        cb.readDefaultParams(tmp_path / "aspAMG.fnames")
    assert e.value.code == -6


def test_reference_parameter_files_if_present(lib):
    from oracle.refdir import reference_file
    fn = reference_file("Tests", "aspAMG.fnames")
    if fn is None:
        pytest.skip("reference tree not mounted")
    p = cb.readDefaultParams(fn)
    assert p.SoC_type == b"DOM" and p.soc_tau == 0.01 and p.nupre == 1 and p.ntv == 6


QR_CALLER = r"""
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>
namespace chronos { void qr_orthonormalize(int n, int k, double *X); }
int main(int argc, char **argv) {
  const int n = std::atoi(argv[1]), k = std::atoi(argv[2]);
  std::vector<double> X((size_t)n * k);
  std::mt19937_64 g(12345);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  for (auto &x : X) x = u(g);
  std::FILE *f = std::fopen(argv[3], "wb");
  std::fwrite(X.data(), sizeof(double), X.size(), f);
  chronos::qr_orthonormalize(n, k, X.data());
  std::fwrite(X.data(), sizeof(double), X.size(), f);
  std::fclose(f);
  return 0;
}
"""


@pytest.mark.parametrize("n,k", [(200000, 6), (70000, 1), (5, 6)])
def test_test_space_qr_thread_independent(lib, tmp_path, n, k):
    """The setup's Householder QR of the test space (threaded over columns
    and rows) gives the same bytes on 1 and 4 threads, orthonormal columns,
    and LAPACK's Q (numpy's QR) to rounding."""
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no C++ compiler")
    src = tmp_path / "qr.cpp"
    src.write_text(QR_CALLER)
    exe = tmp_path / "qr"
    libdir = os.path.join(ROOT, "chronoslab_b200")
    subprocess.run([gxx, "-O2", "-std=c++17", str(src), "-L", libdir, "-lchronos_b200",
                    f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    outs = []
    for threads in ("1", "4"):
        out = tmp_path / f"q{threads}.bin"
        env = dict(os.environ, OMP_NUM_THREADS=threads)
        subprocess.run([str(exe), str(n), str(k), str(out)], check=True, env=env, timeout=300)
        outs.append(out.read_bytes())
    assert outs[0] == outs[1]
    data = np.frombuffer(outs[0], dtype=np.float64)
    X0 = data[:n * k].reshape(k, n).T
    Q = data[n * k:].reshape(k, n).T
    m = min(n, k)
    assert np.allclose(Q[:, :m].T @ Q[:, :m], np.eye(m), atol=1e-12)
    Qn, _ = np.linalg.qr(X0)
    assert np.allclose(Q[:, :m], Qn[:, :m], atol=1e-10)
