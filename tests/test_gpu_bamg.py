"""BAMG prolongation with the per-row work on the GPU (chronos_bamg_device)
against the host restatement (chronos_bamg), which is itself checked against
the reference's BAMG C++ (tests/test_host.py): P's pattern and values and
c_mark equal bit for bit, also when rows outgrow the GPU's per-thread scratch
and are computed on the host, and a setup with the GPU BAMG builds the same
hierarchy and solve as one with the host BAMG."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest
import scipy.sparse as sp

import chronoslab_b200 as cb
from chronoslab_b200 import problems as PB

pytestmark = pytest.mark.gpu


def _same_bamg(A, TV, prm, max_neigh=0):
    fc, nc, S = cb.coarsen(A, prm, 0)
    P, cm = cb.bamg(S, fc, TV, prm)
    Pg, cmg, host_rows = cb.bamg(S, fc, TV, prm, device=True, max_neigh=max_neigh)
    P, Pg = sp.csr_matrix(P), sp.csr_matrix(Pg)
    assert Pg.shape == P.shape
    assert np.array_equal(Pg.indptr, P.indptr) and np.array_equal(Pg.indices, P.indices)
    assert np.array_equal(Pg.data, P.data)
    assert np.array_equal(cmg, cm)
    return host_rows


def _orth(TV):
    Q, _ = np.linalg.qr(np.asarray(TV, dtype=np.float64))
    return Q


@pytest.mark.parametrize("case", ["elasticity", "poisson1", "poisson6", "diffusion"])
def test_bamg_device_matches_host(lib, case):
    rng = np.random.default_rng(4)
    if case == "elasticity":
        A, X = PB.elasticity_q1(9, return_coords=True)
        TV = _orth(PB.rbm_test_space(X))
    elif case == "poisson1":
        A = PB.poisson7(16)
        TV = np.ones((A.shape[0], 1))
    elif case == "poisson6":
        A = PB.poisson7(14)
        TV = _orth(np.column_stack([np.ones(A.shape[0]), rng.random((A.shape[0], 5))]))
    else:
        A = PB.diffusion7(14, sigma=1.0, corr_len=3.0, seed=6)[0]
        TV = _orth(rng.random((A.shape[0], 3)))
    prm = cb.params(ntv=TV.shape[1])
    assert _same_bamg(A, TV, prm) == 0


def test_bamg_device_cubo(lib, cubo):
    """Cubo_4820 with its own test space and the Tests/parm_* prolongation
    (some of its rows have neighbourhoods beyond the GPU's per-thread
    scratch and are computed on the host)."""
    A = cubo["Af"]
    host_rows = _same_bamg(A, _orth(cubo["TV0"]), cb.params())
    assert 0 <= host_rows < 0.01 * A.shape[0]


def test_bamg_rows_beyond_the_gpu_scratch_go_to_the_host(lib):
    """Neighbourhoods of at least four rings (dist_min = 4) of a 7-point grid
    hold up to 129 nodes; with the GPU's per-thread scratch capped at 64
    nodes, those rows are computed on the host, the others on the GPU, and the
    result is still the host's bit for bit."""
    A = PB.poisson7(14)
    rng = np.random.default_rng(2)
    TV = _orth(np.column_stack([np.ones(A.shape[0]), rng.random((A.shape[0], 2))]))
    prm = cb.params(ntv=3, dist_min=4, dist_max=6)
    assert _same_bamg(A, TV, prm, max_neigh=64) > 0
    fc, _, S = cb.coarsen(A, prm, 0)
    with pytest.raises(cb.ChronosError):                # not a power of two
        cb.bamg(S, fc, TV, prm, device=True, max_neigh=100)


def test_setup_with_gpu_bamg_equals_host_bamg(lib):
    """Elasticity 14^3 with the rigid-body test space: the setup's BAMG on the
    GPU (CHRONOS_GPU_BAMG=1) and on the host (the default), each in a child
    process, give the same levels, iterations and solution bit for bit."""
    code = ("import json, numpy as np, chronoslab_b200 as cb;"
            "from chronoslab_b200 import problems as PB;"
            "A, X = PB.elasticity_q1(14, return_coords=True);"
            "TV = PB.rbm_test_space(X); b = PB.elasticity_rhs(A, X, seed=0);"
            "h = cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP64));"
            "x, it, _, fl, _ = h.pcg(b);"
            "print(json.dumps([[h.level_info(l)['n'] for l in range(h.nlevels)], it, fl,"
            " float(x.sum()), x.tobytes().hex()[:4096]]))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = []
    for flag in ("1", "0"):
        env = dict(os.environ, CHRONOS_GPU_BAMG=flag)
        r = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(json.loads(r.stdout.strip().splitlines()[-1]))
    assert outs[0] == outs[1] and outs[0][2] == 0
