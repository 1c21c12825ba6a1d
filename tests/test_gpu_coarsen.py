"""GPU strength of connection (DOM and CLA) and PMIS C/F splitting against the
host splitting and the reference's golden one, bit for bit, through the C ABI."""
import numpy as np
import pytest
import scipy.sparse as sp

import chronoslab_b200 as cb
from chronoslab_b200 import problems as PB

pytestmark = pytest.mark.gpu


def same_split(A, prm, skip=0):
    fc, nc, S = cb.coarsen(A, prm, skip)
    fg, ncg, Sg = cb.coarsen_device(A, prm, skip)
    assert ncg == nc
    assert np.array_equal(fg, fc)
    S, Sg = sp.csr_matrix(S), sp.csr_matrix(Sg)
    assert np.array_equal(Sg.indptr, S.indptr) and np.array_equal(Sg.indices, S.indices)
    return fg, ncg


def test_cubo_golden(lib, cubo, cubo_ref):
    """Cubo_4820 with the Tests/parm_* strength (DOM 0.01): the reference
    run's fcnode."""
    fc, nc = same_split(cubo["Af"], cb.params())
    assert nc == cubo_ref["nc"]
    assert np.array_equal(fc, cubo_ref["fcnode"])


def with_dirichlet(A, rows):
    """A with the given rows and columns replaced by identity ones (columns
    with a single nonzero: the PMIS marks them fine from the start)."""
    A = sp.lil_matrix(A)
    for r in rows:
        A[r, :] = 0.0
        A[:, r] = 0.0
        A[r, r] = 1.0
    A = sp.csr_matrix(A)
    A.eliminate_zeros()
    A.sort_indices()
    return A


def _case(case):
    if case == "elasticity":
        return PB.elasticity_q1(7)
    if case == "poisson":
        return PB.poisson7(14)
    if case == "diffusion":
        return PB.diffusion7(12, sigma=1.0, corr_len=3.0, seed=4)[0]
    if case == "nonneg":                 # every off-diagonal entry >= 0: CLA's |a| branch
        A = abs(PB.poisson7(10)).tocsr()
        A.sort_indices()
        return A
    return with_dirichlet(PB.poisson7(9), [0, 5, 17, 300, 728])


@pytest.mark.parametrize("soc", ["DOM", "CLA"])
@pytest.mark.parametrize("case", ["elasticity", "poisson", "diffusion", "dirichlet", "nonneg"])
@pytest.mark.parametrize("tau", [0.01, 0.25])
def test_matches_host(lib, case, tau, soc):
    A = _case(case)
    for skip in (0, 37):
        same_split(A, cb.params(SoC_type=soc, soc_tau=tau), skip)


def test_empty_strength(lib):
    """tau above every strength (the diagonal's is 1): S is empty, no node has
    a neighbour, and every node turns coarse in the first round."""
    A = PB.poisson7(6)
    fc, nc = same_split(A, cb.params(SoC_type="DOM", soc_tau=2.0))
    assert nc == A.shape[0]


def test_cla_setup_on_the_gpu_matches_host_coarsening(lib):
    """A hierarchy with CLA strength (tau 0.25, as FlowCLAS_0.m) coarsens on the
    GPU by default and on the host with CHRONOS_GPU_COARSEN=0 in a child
    process: the same level sizes and the same PCG_CJ iterations."""
    import json
    import os
    import subprocess
    import sys
    code = ("import json, numpy as np, chronoslab_b200 as cb;"
            "from chronoslab_b200 import problems as PB;"
            "A = PB.diffusion7(20, sigma=1.0, corr_len=4.0, seed=2)[0];"
            "b = PB.uniform_rhs(A.shape[0], seed=3);"
            "h = cb.Hierarchy(A, np.ones(A.shape[0]), cb.params(SoC_type='CLA', soc_tau=0.25, ntv=1));"
            "x, it, _, fl, _ = h.pcg(b);"
            "print(json.dumps([[h.level_info(l)['n'] for l in range(h.nlevels)], it, fl]))")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = []
    for flag in ("1", "0"):
        env = dict(os.environ, CHRONOS_GPU_COARSEN=flag)
        r = subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(json.loads(r.stdout.strip().splitlines()[-1]))
    assert outs[0] == outs[1] and outs[0][2] == 0


def test_hierarchy_levels_match_host_split(lib):
    """The setup's first coarse level has the size of the host splitting."""
    A, X = PB.elasticity_q1(8, return_coords=True)
    TV = PB.rbm_test_space(X)
    _, nc, _ = cb.coarsen(A, cb.params(), 0)        # six test vectors given: no draws
    with cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP32)) as h:
        assert h.level_info(1)["n"] == nc
