"""Differentiable AMG-PCG solve: a torch.autograd.Function over the C ABI.

forward:  u = A(values)^{-1} b by the GPU PCG (hierarchy built for A)
backward: the adjoint solve A lambda = dJ/du on the same hierarchy (A is SPD,
          so A^T = A), then dJ/dA_ij = -lambda_i u_j on A's pattern
          (chronos_adjoint_grad, one scatter kernel) and dJ/db = lambda.

Gradients with respect to matrix *values* chain through any torch code that
assembles them; diffusion_values() assembles the 7-point finite-volume
diffusion operator of problems.diffusion_from_logk from a log-coefficient
field, so dJ/dlog k follows by autograd.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import torch

from . import CHRONOS_FP32, Hierarchy, params


class AMGSolve(torch.autograd.Function):
    """u = AMGSolve.apply(values, b, indptr, indices, prm, itmax, tol)."""

    @staticmethod
    def forward(ctx, values, b, indptr, indices, prm, itmax, tol):
        n = indptr.size - 1
        A = sp.csr_matrix((values.detach().cpu().numpy().astype(np.float64), indices, indptr),
                          shape=(n, n))
        h = Hierarchy(A, np.ones(n), prm)          # constant near-null vector
        u, it, rv, flag, _ = h.pcg(b.detach().cpu().numpy().astype(np.float64), itmax=itmax,
                                   tol=tol)
        if flag != 0:
            raise RuntimeError(f"PCG did not reach {tol} in {itmax} iterations")
        ctx.h, ctx.itmax, ctx.tol = h, itmax, tol
        ctx.u = u
        return torch.from_numpy(u).to(values.device)

    @staticmethod
    def backward(ctx, grad_u):
        g = grad_u.detach().cpu().numpy().astype(np.float64)
        lam, grad_vals, it = ctx.h.adjoint_grad(ctx.u, g, ctx.itmax, ctx.tol)
        ctx.h.close()
        dev = grad_u.device
        return (torch.from_numpy(grad_vals).to(dev), torch.from_numpy(lam).to(dev),
                None, None, None, None, None)


def solve(values, b, indptr, indices, prm=None, itmax=2000, tol=1e-12):
    prm = prm or params(precision=CHRONOS_FP32, ntv=1)
    return AMGSolve.apply(values, b, np.ascontiguousarray(indptr, np.int32),
                          np.ascontiguousarray(indices, np.int32), prm, itmax, tol)


# ---------------------------------------------------------------------------
# differentiable diffusion assembly (same operator and CSR order as
# problems.diffusion_from_logk)
# ---------------------------------------------------------------------------

class DiffusionPattern:
    """CSR pattern of the nz x ny x nx 7-point operator and the map from its
    COO assembly order to CSR positions."""

    def __init__(self, shape, zaniso=0.01):
        nz, ny, nx = shape
        self.shape, self.zaniso = shape, zaniso
        n = nx * ny * nz
        idx = np.arange(n).reshape(nz, ny, nx)
        rows = np.concatenate([idx.ravel(), idx[:, :, :-1].ravel(), idx[:, :, 1:].ravel(),
                               idx[:, :-1, :].ravel(), idx[:, 1:, :].ravel(),
                               idx[:-1, :, :].ravel(), idx[1:, :, :].ravel()])
        cols = np.concatenate([idx.ravel(), idx[:, :, 1:].ravel(), idx[:, :, :-1].ravel(),
                               idx[:, 1:, :].ravel(), idx[:, :-1, :].ravel(),
                               idx[1:, :, :].ravel(), idx[:-1, :, :].ravel()])
        M = sp.csr_matrix((np.arange(1, rows.size + 1, dtype=np.float64), (rows, cols)),
                          shape=(n, n))
        M.sort_indices()
        self.indptr = M.indptr.astype(np.int32)
        self.indices = M.indices.astype(np.int32)
        pos = np.empty(rows.size, dtype=np.int64)
        pos[M.data.astype(np.int64) - 1] = np.arange(M.nnz)
        self.pos = torch.from_numpy(pos)
        self.n, self.nnz = n, M.nnz


def diffusion_values(logk, pat: DiffusionPattern):
    """CSR values of the diffusion operator (torch, differentiable in logk,
    shape (nz, ny, nx))."""
    z = pat.zaniso
    k = torch.exp(logk)
    hm = lambda a, b: 2.0 * a * b / (a + b)
    tx = hm(k[:, :, :-1], k[:, :, 1:])
    ty = hm(k[:, :-1, :], k[:, 1:, :])
    tz = z * hm(k[:-1, :, :], k[1:, :, :])
    diag = torch.zeros_like(k)
    diag = diag + torch.nn.functional.pad(tx, (0, 1)) + torch.nn.functional.pad(tx, (1, 0))
    diag = diag + torch.nn.functional.pad(ty, (0, 0, 0, 1)) + torch.nn.functional.pad(ty, (0, 0, 1, 0))
    diag = diag + torch.nn.functional.pad(tz, (0, 0, 0, 0, 0, 1)) + \
        torch.nn.functional.pad(tz, (0, 0, 0, 0, 1, 0))
    bnd = torch.zeros_like(k)
    bnd[:, :, 0] += 2 * k[:, :, 0]
    bnd[:, :, -1] += 2 * k[:, :, -1]
    bnd[:, 0, :] += 2 * k[:, 0, :]
    bnd[:, -1, :] += 2 * k[:, -1, :]
    bnd[0, :, :] += 2 * z * k[0, :, :]
    bnd[-1, :, :] += 2 * z * k[-1, :, :]
    diag = diag + bnd
    coo = torch.cat([diag.reshape(-1), -tx.reshape(-1), -tx.reshape(-1), -ty.reshape(-1),
                     -ty.reshape(-1), -tz.reshape(-1), -tz.reshape(-1)])
    out = torch.zeros(pat.nnz, dtype=coo.dtype, device=coo.device)
    return out.index_add(0, pat.pos.to(coo.device), coo)
