"""Seeded synthetic SPD problems standing in for the solve path's workloads.

The reference ships no problem generators (only .mat fixtures), so these build
the matrices named by the benchmark configurations, deterministically from a
seed, as 0-based CSR (scipy.sparse.csr_matrix, sorted columns, FP64):

  poisson7(nx)              7-point finite-difference Laplacian, Dirichlet
                            boundary eliminated (nx^3 unknowns).
  elasticity_q1(ne)         trilinear hex (Q1) linear elasticity on the unit
                            cube with ne^3 elements, E = 1, nu = 0.3, clamped at
                            z = 0 (those DOFs eliminated); 3 DOF per node.
  diffusion7(nx, ...)       7-point finite-volume diffusion with a seeded
                            log-normal coefficient exp(s*g), g a Gaussian field
                            of given correlation length, z-faces scaled by an
                            anisotropy factor; Dirichlet boundary eliminated.
  rbm_test_space(coords)    the six rigid-body modes (mk_rbm_3d.m) of the
                            elasticity nodes.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _lap1(m):
    return sp.diags([-np.ones(m - 1), 2.0 * np.ones(m), -np.ones(m - 1)], [-1, 0, 1])


def poisson7(nx, ny=None, nz=None):
    ny = ny or nx
    nz = nz or nx
    Ix, Iy, Iz = sp.identity(nx), sp.identity(ny), sp.identity(nz)
    A = (sp.kron(Iz, sp.kron(Iy, _lap1(nx))) + sp.kron(Iz, sp.kron(_lap1(ny), Ix))
         + sp.kron(_lap1(nz), sp.kron(Iy, Ix))).tocsr()
    A.sum_duplicates()
    A.sort_indices()
    return A


# ---------------------------------------------------------------------------
# Q1 elasticity
# ---------------------------------------------------------------------------

def q1_element_stiffness(h, E=1.0, nu=0.3):
    """24x24 stiffness of a cube element of edge h (2x2x2 Gauss), local node
    a = ax + 2*ay + 4*az with ax,ay,az in {0,1}, DOF order (node, x/y/z)."""
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] += 2 * mu
    D[3:, 3:] = np.diag([mu, mu, mu])
    corners = np.array([[a & 1, (a >> 1) & 1, (a >> 2) & 1] for a in range(8)], dtype=float)
    g = 0.5 / np.sqrt(3.0)
    K = np.zeros((24, 24))
    for qx in (0.5 - g, 0.5 + g):
        for qy in (0.5 - g, 0.5 + g):
            for qz in (0.5 - g, 0.5 + g):
                q = np.array([qx, qy, qz])
                dN = np.zeros((8, 3))            # d N_a / d xi (reference cube [0,1]^3)
                for a in range(8):
                    c = corners[a]
                    f = np.where(c == 1, q, 1 - q)
                    s = np.where(c == 1, 1.0, -1.0)
                    dN[a] = [s[0] * f[1] * f[2], f[0] * s[1] * f[2], f[0] * f[1] * s[2]]
                dN /= h
                B = np.zeros((6, 24))
                for a in range(8):
                    bx, by, bz = dN[a]
                    B[0, 3 * a] = bx
                    B[1, 3 * a + 1] = by
                    B[2, 3 * a + 2] = bz
                    B[3, 3 * a] = by; B[3, 3 * a + 1] = bx
                    B[4, 3 * a + 1] = bz; B[4, 3 * a + 2] = by
                    B[5, 3 * a] = bz; B[5, 3 * a + 2] = bx
                K += B.T @ D @ B * (h ** 3) / 8.0
    return 0.5 * (K + K.T)


def elasticity_q1(ne, E=1.0, nu=0.3, return_coords=False):
    """Assembled per node from the 27-point stencil of the uniform mesh: the
    3x3 block coupling node a to node a+off is the sum, over the (up to 8)
    elements containing both, of the element-matrix block."""
    h = 1.0 / ne
    Ke = q1_element_stiffness(h, E, nu)
    nn1 = ne + 1
    nodes = np.arange(nn1 ** 3)
    iz, rem = np.divmod(nodes, nn1 * nn1)
    iy, ix = np.divmod(rem, nn1)
    free = iz > 0                                   # clamped at z = 0
    fid = -np.ones(nn1 ** 3, dtype=np.int64)
    fid[free] = np.arange(int(free.sum()))
    nfree = int(free.sum())
    offs = [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
    # Block values per (node, offset): [nnodes, 27, 3, 3]
    fn = np.flatnonzero(free)
    fx, fy, fz = ix[fn], iy[fn], iz[fn]
    blocks = np.zeros((fn.size, 27, 3, 3))
    valid = np.zeros((fn.size, 27), dtype=bool)
    for o, (dx, dy, dz) in enumerate(offs):
        nx_, ny_, nz_ = fx + dx, fy + dy, fz + dz
        inside = (nx_ >= 0) & (nx_ <= ne) & (ny_ >= 0) & (ny_ <= ne) & (nz_ >= 1) & (nz_ <= ne)
        for sx in (0, 1):
            for sy in (0, 1):
                for sz in (0, 1):
                    # element whose local corner (sx,sy,sz) is this node
                    ex, ey, ez = fx - sx, fy - sy, fz - sz
                    ok = (ex >= 0) & (ex < ne) & (ey >= 0) & (ey < ne) & (ez >= 0) & (ez < ne)
                    lx, ly, lz = sx + dx, sy + dy, sz + dz
                    if not (0 <= lx <= 1 and 0 <= ly <= 1 and 0 <= lz <= 1):
                        continue
                    a = sx + 2 * sy + 4 * sz
                    b = lx + 2 * ly + 4 * lz
                    m = ok & inside
                    blocks[m, o] += Ke[3 * a:3 * a + 3, 3 * b:3 * b + 3]
                    valid[m, o] |= True
    # Column node ids per offset (increasing in offset order -> sorted columns)
    cols_node = np.zeros((fn.size, 27), dtype=np.int64)
    for o, (dx, dy, dz) in enumerate(offs):
        nx_, ny_, nz_ = fx + dx, fy + dy, fz + dz
        inside = (nx_ >= 0) & (nx_ <= ne) & (ny_ >= 0) & (ny_ <= ne) & (nz_ >= 1) & (nz_ <= ne)
        g = np.where(inside, nx_ + nn1 * (ny_ + nn1 * nz_), 0)
        cols_node[:, o] = np.where(inside, fid[g], -1)
    valid &= cols_node >= 0
    cnt_nodes = valid.sum(axis=1)                    # neighbour nodes per node
    row_len = 3 * cnt_nodes                          # per DOF row
    n = 3 * nfree
    indptr = np.zeros(n + 1, dtype=np.int64)
    indptr[1:] = np.cumsum(np.repeat(row_len, 3))
    # entries: for node r, dof i: for each valid offset o (ascending), dof j
    vb = valid[:, :, None, None] & np.ones((1, 1, 3, 3), dtype=bool)
    # reorder to [node, i, o, j]
    vals = np.transpose(blocks, (0, 2, 1, 3))
    msk = np.transpose(vb, (0, 2, 1, 3))
    colsf = (3 * cols_node[:, None, :, None] + np.arange(3)[None, None, None, :])
    colsf = np.broadcast_to(colsf, vals.shape)
    data = vals[msk]
    indices = colsf[msk]
    A = sp.csr_matrix((data, indices.astype(np.int32), indptr), shape=(n, n))
    A.sort_indices()
    if return_coords:
        coords = np.stack([fx * h, fy * h, fz * h], axis=1)
        return A, coords
    return A


def rbm_test_space(coords):
    """mk_rbm_3d.m:1-27: six rigid-body modes, 3 DOF per node (x,y,z)."""
    nn = coords.shape[0]
    R = np.zeros((3 * nn, 6))
    R[0::3, 0] = 1
    R[1::3, 1] = 1
    R[2::3, 2] = 1
    XB = coords.sum(axis=0) / nn
    R[1::3, 3] = -coords[:, 2] + XB[2]
    R[2::3, 3] = coords[:, 1] - XB[1]
    R[0::3, 4] = coords[:, 2] - XB[2]
    R[2::3, 4] = -coords[:, 0] + XB[0]
    R[0::3, 5] = -coords[:, 1] + XB[1]
    R[1::3, 5] = coords[:, 0] - XB[0]
    return R


def elasticity_rhs(A, coords, seed, noise=0.01):
    """Unit body force (z component) plus seeded N(0, noise^2) noise."""
    n = A.shape[0]
    rng = np.random.default_rng(seed)
    b = np.zeros(n)
    b[2::3] = 1.0 / coords.shape[0]
    return b + noise * rng.standard_normal(n) / coords.shape[0]


# ---------------------------------------------------------------------------
# Heterogeneous diffusion
# ---------------------------------------------------------------------------

def gaussian_field(shape, corr_len, seed):
    """Zero-mean, unit-variance Gaussian field with Gaussian covariance of
    correlation length corr_len (cells), by FFT filtering of white noise."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape)
    k = [np.fft.fftfreq(s) for s in shape]
    K2 = sum(np.meshgrid(*[kk ** 2 for kk in k], indexing="ij"))
    filt = np.exp(-0.5 * (2 * np.pi) ** 2 * K2 * corr_len ** 2 / 2.0)
    g = np.real(np.fft.ifftn(np.fft.fftn(w) * filt))
    g -= g.mean()
    s = g.std()
    return g / s if s > 0 else g


def diffusion7(nx, sigma=2.0, corr_len=8.0, zaniso=0.01, seed=0, logk=None):
    """Cell-centred finite volumes on nx^3 unit-spaced cells, coefficient
    k = exp(sigma*g); face transmissibility = harmonic mean of the two cells'
    k (z faces times zaniso); Dirichlet (zero) boundary through half-cell
    transmissibility 2k.  Returns (A, logk)."""
    shape = (nx, nx, nx)   # (z, y, x) indexing, x fastest
    if logk is None:
        logk = sigma * gaussian_field(shape, corr_len, seed)
    k = np.exp(logk)
    return diffusion_from_logk(logk, zaniso), logk


def face_transmissibilities(logk, zaniso):
    k = np.exp(logk)
    hm = lambda a, b: 2.0 * a * b / (a + b)
    tx = hm(k[:, :, :-1], k[:, :, 1:])
    ty = hm(k[:, :-1, :], k[:, 1:, :])
    tz = zaniso * hm(k[:-1, :, :], k[1:, :, :])
    return tx, ty, tz


def diffusion_from_logk(logk, zaniso=0.01):
    nz, ny, nx = logk.shape
    k = np.exp(logk)
    tx, ty, tz = face_transmissibilities(logk, zaniso)
    n = nx * ny * nz
    idx = np.arange(n).reshape(nz, ny, nx)
    diag = np.zeros((nz, ny, nx))
    diag[:, :, :-1] += tx; diag[:, :, 1:] += tx
    diag[:, :-1, :] += ty; diag[:, 1:, :] += ty
    diag[:-1, :, :] += tz; diag[1:, :, :] += tz
    # Dirichlet boundary faces: transmissibility 2k to the boundary value 0
    diag[:, :, 0] += 2 * k[:, :, 0]; diag[:, :, -1] += 2 * k[:, :, -1]
    diag[:, 0, :] += 2 * k[:, 0, :]; diag[:, -1, :] += 2 * k[:, -1, :]
    diag[0, :, :] += 2 * zaniso * k[0, :, :]; diag[-1, :, :] += 2 * zaniso * k[-1, :, :]
    rows = [idx.ravel(), idx[:, :, :-1].ravel(), idx[:, :, 1:].ravel(),
            idx[:, :-1, :].ravel(), idx[:, 1:, :].ravel(),
            idx[:-1, :, :].ravel(), idx[1:, :, :].ravel()]
    cols = [idx.ravel(), idx[:, :, 1:].ravel(), idx[:, :, :-1].ravel(),
            idx[:, 1:, :].ravel(), idx[:, :-1, :].ravel(),
            idx[1:, :, :].ravel(), idx[:-1, :, :].ravel()]
    vals = [diag.ravel(), -tx.ravel(), -tx.ravel(), -ty.ravel(), -ty.ravel(),
            -tz.ravel(), -tz.ravel()]
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    return A


def uniform_rhs(n, seed, ncols=1):
    rng = np.random.default_rng(seed)
    if ncols == 1:
        return rng.uniform(-1.0, 1.0, n)
    return rng.uniform(-1.0, 1.0, (n, ncols))
