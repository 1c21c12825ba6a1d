"""Block of right-hand sides (SpMM V-cycles, per-column PCG_CJ recurrences)
against single-column solves and the oracle, on the heterogeneous diffusion
problem (log-normal coefficient exp(2g), 100:1 z-anisotropy)."""
import numpy as np
import pytest

import chronoslab_b200 as cb
from chronoslab_b200 import problems as PB
from oracle import amg_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def diffusion():
    A, _ = PB.diffusion7(24, sigma=2.0, corr_len=8.0, zaniso=0.01, seed=5)
    B = PB.uniform_rhs(A.shape[0], seed=6, ncols=16)
    return A, B


@pytest.mark.parametrize("prec", [cb.CHRONOS_FP64, cb.CHRONOS_FP32])
def test_block_matches_columns(lib, diffusion, prec):
    A, B = diffusion
    with cb.Hierarchy(A, np.ones(A.shape[0]),cb.params(precision=prec, ntv=1)) as h:
        X, its, flags, sec = h.pcg_block(B, itmax=1000, tol=1e-8)
        assert np.all(flags == 0)
        for j in range(B.shape[1]):
            x, it, _, flag, _ = h.pcg(B[:, j], itmax=1000, tol=1e-8)
            assert flag == 0 and abs(int(its[j]) - it) <= 1
            assert np.linalg.norm(X[:, j] - x) <= 1e-6 * np.linalg.norm(x)
            assert np.linalg.norm(B[:, j] - A @ X[:, j]) <= 1e-8 * np.linalg.norm(B[:, j])


def test_block_iterations_match_oracle(lib, diffusion):
    A, B = diffusion
    with cb.Hierarchy(A, np.ones(A.shape[0]),cb.params(precision=cb.CHRONOS_FP64, ntv=1)) as h:
        parts = []
        for l in range(h.nlevels):
            p = {"A": h.export(l, "A")}
            if l < h.nlevels - 1:
                p.update(G=h.export(l, "G"), P=h.export(l, "P"), omega=h.level_info(l)["omega"])
            parts.append(p)
        Ho = O.hierarchy_from_parts(parts)
        X, its, flags, _ = h.pcg_block(B[:, :4], itmax=1000, tol=1e-8)
        for j in range(4):
            _, ito, _, _ = O.pcg_cj(lambda r: O.amg_vcycle(Ho, r), lambda v: A @ v, B[:, j],
                                    np.zeros(A.shape[0]), 1000, 1e-8)
            assert abs(int(its[j]) - ito) <= 1


def test_block_padding_and_zero_columns(lib, diffusion):
    A, B = diffusion
    B5 = B[:, :5].copy()
    B5[:, 2] = 0.0
    with cb.Hierarchy(A, np.ones(A.shape[0]),cb.params(ntv=1)) as h:
        X, its, flags, _ = h.pcg_block(B5, itmax=1000, tol=1e-8)
        assert X.shape == B5.shape
        assert its[2] == 0 and flags[2] == 0 and not np.any(X[:, 2])
        for j in (0, 1, 3, 4):
            assert flags[j] == 0
            assert np.linalg.norm(B5[:, j] - A @ X[:, j]) <= 1e-8 * np.linalg.norm(B5[:, j])
        # more than 16 columns: solved in chunks of 16
        B20 = np.concatenate([B, B[:, :4]], axis=1)
        X20, its20, fl20, _ = h.pcg_block(B20, itmax=1000, tol=1e-8)
        assert np.all(fl20 == 0) and np.array_equal(its20[16:], its20[:4])


def test_block_host_loop_matches_graph_loop(lib, diffusion):
    """The per-iteration graph launched from a host loop (use_graph = 0, what
    a profiler sees) gives the conditional-graph loop's results bit for bit."""
    A, B = diffusion
    out = []
    for g in (1, 0):
        with cb.Hierarchy(A, np.ones(A.shape[0]), cb.params(precision=cb.CHRONOS_FP32, ntv=1,
                                                            use_graph=g)) as h:
            X, its, flags, _ = h.pcg_block(B[:, :5], itmax=1000, tol=1e-8)
            out.append((X, its, flags))
    assert np.array_equal(out[0][1], out[1][1]) and np.all(out[1][2] == 0)
    assert np.array_equal(out[0][0], out[1][0])
