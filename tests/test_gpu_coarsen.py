"""GPU strength of connection (DOM) and PMIS C/F splitting against the host
splitting and the reference's golden one, bit for bit, through the C ABI."""
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


@pytest.mark.parametrize("case", ["elasticity", "poisson", "diffusion", "dirichlet"])
@pytest.mark.parametrize("tau", [0.01, 0.25])
def test_matches_host(lib, case, tau):
    if case == "elasticity":
        A = PB.elasticity_q1(7)
    elif case == "poisson":
        A = PB.poisson7(14)
    elif case == "diffusion":
        A = PB.diffusion7(12, sigma=1.0, corr_len=3.0, seed=4)[0]
    else:
        A = with_dirichlet(PB.poisson7(9), [0, 5, 17, 300, 728])
    for skip in (0, 37):
        same_split(A, cb.params(SoC_type="DOM", soc_tau=tau), skip)


def test_empty_strength(lib):
    """tau above every strength (the diagonal's is 1): S is empty, no node has
    a neighbour, and every node turns coarse in the first round."""
    A = PB.poisson7(6)
    fc, nc = same_split(A, cb.params(SoC_type="DOM", soc_tau=2.0))
    assert nc == A.shape[0]


def test_cla_is_not_on_the_gpu(lib):
    A = PB.poisson7(6)
    with pytest.raises(cb.ChronosError):
        cb.coarsen_device(A, cb.params(SoC_type="CLA", soc_tau=0.25))


def test_hierarchy_levels_match_host_split(lib):
    """The setup's first coarse level has the size of the host splitting."""
    A, X = PB.elasticity_q1(8, return_coords=True)
    TV = PB.rbm_test_space(X)
    _, nc, _ = cb.coarsen(A, cb.params(), 0)        # six test vectors given: no draws
    with cb.Hierarchy(A, TV, cb.params(precision=cb.CHRONOS_FP32)) as h:
        assert h.level_info(1)["n"] == nc
