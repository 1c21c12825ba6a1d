"""Adjoint gradients of J(u) = 1/2 ||u - u*||^2, u = A(log k)^{-1} b, for the
log-normal diffusion problem: the GPU adjoint (same hierarchy, scatter of
-lambda_i u_j on A's pattern) against central finite differences and against
the gradient of a plain FP64 direct solve."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

import chronoslab_b200 as cb
from chronoslab_b200 import problems as PB
from chronoslab_b200.autodiff import DiffusionPattern, diffusion_values, solve


def direct_solver(A):
    lu = spla.splu(A.tocsc())
    return lu.solve


def oracle_solver(A):
    """FP64 PCG_CJ of the oracle (C/OpenMP) with its own FP64 hierarchy built
    with the reference's FSAI/BAMG C++, to 1e-13."""
    from oracle import amg_oracle as O
    from oracle import c_oracle as CO
    if not O.ref_available():
        pytest.skip("oracle/_ref not built")
    prm = O.default_params()
    prm["tspace"]["ntv"] = 1
    CH = CO.CHierarchy(CO.reference_hierarchy(A, None, prm))

    def s(rhs):
        x, it, rv, flag = CH.pcg(rhs, itmax=5000, tol=1e-13)
        assert flag == 0
        return x
    return s


def fp64_reference_grad(logk, pat, b, ustar, make_solver=direct_solver):
    """dJ/dlogk with an FP64 solve and the same assembly (torch)."""
    lk = torch.from_numpy(logk).requires_grad_(True)
    vals = diffusion_values(lk, pat)
    A = sp.csr_matrix((vals.detach().numpy(), pat.indices, pat.indptr), shape=(pat.n, pat.n))
    slv = make_solver(A)
    u = slv(b)
    lam = slv(u - ustar)
    rows = np.repeat(np.arange(pat.n), np.diff(pat.indptr))
    gvals = -lam[rows] * u[pat.indices]
    vals.backward(torch.from_numpy(gvals))
    return lk.grad.numpy(), 0.5 * float(np.sum((u - ustar) ** 2))


def test_diffusion_values_match_assembly():
    logk = PB.gaussian_field((5, 6, 7), 2.0, seed=3)
    A = PB.diffusion_from_logk(logk, 0.01)
    pat = DiffusionPattern(logk.shape, 0.01)
    v = diffusion_values(torch.from_numpy(logk), pat).numpy()
    assert np.array_equal(pat.indptr, A.indptr) and np.array_equal(pat.indices, A.indices)
    assert np.allclose(v, A.data, rtol=1e-14, atol=0)


def test_adjoint_formula_against_fd_cpu():
    """The chain rule (scatter -lambda_i u_j, then autograd through the
    assembly) against central differences, all in FP64 on the CPU."""
    rng = np.random.default_rng(0)
    shape = (4, 5, 6)
    logk = PB.gaussian_field(shape, 2.0, seed=1)
    pat = DiffusionPattern(shape, 0.01)
    b = rng.uniform(-1, 1, pat.n)
    ustar = rng.uniform(-1, 1, pat.n) * 0.1
    g, _ = fp64_reference_grad(logk, pat, b, ustar)

    def J(lk):
        v = diffusion_values(torch.from_numpy(lk), pat).numpy()
        A = sp.csr_matrix((v, pat.indices, pat.indptr), shape=(pat.n, pat.n))
        u = spla.spsolve(A.tocsc(), b)
        return 0.5 * np.sum((u - ustar) ** 2)
    h = 1e-6
    for _ in range(8):
        d = rng.standard_normal(shape)
        fd = (J(logk + h * d) - J(logk - h * d)) / (2 * h)
        assert abs(fd - np.sum(g * d)) <= 1e-6 * max(abs(fd), 1e-12)


@pytest.mark.gpu
def test_adjoint_fd_gpu(lib):
    """GPU forward/adjoint solves vs central finite differences (h = 1e-6,
    32 seeded directions), relative error <= 1e-6 (C5 protocol, 16^3 grid)."""
    rng = np.random.default_rng(7)
    shape = (16, 16, 16)
    logk = PB.gaussian_field(shape, 4.0, seed=2)                 # sigma = 1
    pat = DiffusionPattern(shape, 0.01)
    b = rng.uniform(-1, 1, pat.n)
    logk_star = logk + 0.1 * PB.gaussian_field(shape, 4.0, seed=3)
    vstar = diffusion_values(torch.from_numpy(logk_star), pat)
    ustar = solve(vstar, torch.from_numpy(b), pat.indptr, pat.indices).numpy()
    prm = cb.params(precision=cb.CHRONOS_FP64, ntv=1)

    def J_and_grad(lk, need_grad):
        t = torch.from_numpy(lk).requires_grad_(need_grad)
        u = solve(diffusion_values(t, pat), torch.from_numpy(b), pat.indptr, pat.indices,
                  prm=prm, tol=1e-14, itmax=4000)
        J = 0.5 * torch.sum((u - torch.from_numpy(ustar)) ** 2)
        if need_grad:
            J.backward()
            return J.item(), t.grad.numpy()
        return J.item(), None

    J0, g = J_and_grad(logk, True)
    h = 1e-6
    errs = []
    for _ in range(32):
        d = rng.standard_normal(shape)
        fd = (J_and_grad(logk + h * d, False)[0] - J_and_grad(logk - h * d, False)[0]) / (2 * h)
        errs.append(abs(fd - np.sum(g * d)) / max(abs(fd), 1e-300))
    assert max(errs) <= 1e-6, max(errs)


@pytest.mark.gpu
def test_adjoint_vs_fp64_reference_gradient(lib):
    """FP32-hierarchy GPU adjoint gradient vs the plain FP64 direct-solve
    gradient on the C5 grid (64^3, sigma = 1)."""
    rng = np.random.default_rng(11)
    shape = (64, 64, 64)
    logk = PB.gaussian_field(shape, 8.0, seed=5)
    pat = DiffusionPattern(shape, 0.01)
    b = rng.uniform(-1, 1, pat.n)
    ustar = rng.uniform(-1, 1, pat.n) * 0.01
    g_ref, J_ref = fp64_reference_grad(logk, pat, b, ustar, oracle_solver)
    t = torch.from_numpy(logk).requires_grad_(True)
    u = solve(diffusion_values(t, pat), torch.from_numpy(b), pat.indptr, pat.indices,
              prm=cb.params(precision=cb.CHRONOS_FP32, ntv=1), tol=1e-12, itmax=4000)
    J = 0.5 * torch.sum((u - torch.from_numpy(ustar)) ** 2)
    J.backward()
    assert abs(J.item() - J_ref) <= 1e-9 * J_ref
    assert np.linalg.norm(t.grad.numpy() - g_ref) <= 1e-6 * np.linalg.norm(g_ref)
