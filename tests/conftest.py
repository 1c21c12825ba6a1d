"""Shared fixtures.  Tests marked `gpu` need a CUDA device; everything else runs
on the CPU (the C ABI library loads without a GPU, and its host-side setup
entry points run there)."""
import json
import os
import sys

import numpy as np
import pytest
import scipy.sparse as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def lib():
    from chronoslab_b200 import build
    build.build()
    from chronoslab_b200 import _lib
    return _lib.load()


@pytest.fixture(scope="session")
def cubo():
    """Cubo_4820 with computeAMG's Dirichlet-diagonal fix (golden value)."""
    z = np.load(os.path.join(GOLDEN, "cubo_A_upper.npz"))
    n = int(z["n"])
    U = sp.csr_matrix((z["data"], z["indices"], z["indptr"]), shape=(n, n))
    A = (U + sp.triu(U, 1).T).tocsr()
    A.sort_indices()
    Af = A.copy()
    d = Af.diagonal()
    d[d == 1.0] = float(z["diag_fix"])
    Af.setdiag(d)
    Af.sort_indices()
    return {"A": A, "Af": Af, "TV0": z["TV0"], "n": n}


def load_csr(z, key):
    shape = tuple(int(s) for s in z[key + "_shape"])
    return sp.csr_matrix((z[key + "_data"], z[key + "_indices"], z[key + "_indptr"]), shape=shape)


@pytest.fixture(scope="session")
def cubo_ref():
    with open(os.path.join(GOLDEN, "cubo_ref.json")) as f:
        info = json.load(f)
    fz = np.load(os.path.join(GOLDEN, "cubo_ref_fsai.npz"))
    bz = np.load(os.path.join(GOLDEN, "cubo_ref_bamg.npz"))
    return {"info": info, "G": load_csr(fz, "G"), "P": load_csr(bz, "P"),
            "fcnode": bz["fcnode"].astype(np.int64), "nc": int(bz["nc"]),
            "c_mark": bz["c_mark"].astype(np.int64)}


@pytest.fixture(scope="session")
def small_ref():
    z = np.load(os.path.join(GOLDEN, "small_ref.npz"))
    return {k: load_csr(z, k) for k in ("Ap", "Gp", "Ae", "Ge")}


def rowwise_close(G, Gref, tol):
    """Same pattern, and every entry within tol of its row's largest magnitude
    (FSAI rows may hold exact zeros where A stores structural zeros)."""
    assert np.array_equal(G.indptr, Gref.indptr) and np.array_equal(G.indices, Gref.indices)
    rows = np.repeat(np.arange(Gref.shape[0]), np.diff(Gref.indptr))
    scale = np.zeros(Gref.shape[0])
    np.maximum.at(scale, rows, np.abs(Gref.data))
    err = np.abs(np.asarray(G.data) - Gref.data) / np.maximum(scale[rows], 1e-300)
    return float(err.max()) <= tol


def ref_available():
    from oracle import amg_oracle as O
    return O.ref_available()
