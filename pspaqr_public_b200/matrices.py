"""Synthetic sparse matrices and right-hand sides for the pspaQR workloads.

The reference ships no matrices (its run scripts point at Matrix Market files
that are not part of the repository), so every workload is generated here.
Node numbering follows the tensor coordinates of ``linspace_nd``
(util.cpp:901-930): grid point ``(i0, i1, ..., i_{d-1})`` is unknown
``i0*n^(d-1) + ... + i_{d-1}``.  All grids use Dirichlet boundaries: only the
``n^d`` interior points are unknowns and couplings to the boundary are dropped.

Matrices are returned as CSC triples ``(colptr, rowidx, values)`` with sorted
row indices, 0-based, int32 / float64 -- the layout the C ABI takes.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _grid_shift_pairs(n: int, d: int):
    """Yield (p, q, axis) index arrays of all nearest-neighbour pairs p<q."""
    idx = np.arange(n ** d, dtype=np.int64).reshape((n,) * d)
    for ax in range(d):
        sl_lo = [slice(None)] * d
        sl_hi = [slice(None)] * d
        sl_lo[ax] = slice(0, n - 1)
        sl_hi[ax] = slice(1, n)
        yield idx[tuple(sl_lo)].ravel(), idx[tuple(sl_hi)].ravel(), ax


def _to_csc(A: sp.spmatrix):
    A = sp.csc_matrix(A)
    A.sum_duplicates()
    A.sort_indices()
    return (A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64))


def laplacian(n: int, d: int):
    """Negative Laplacian, (2d+1)-point stencil: 2d on the diagonal, -1 off it."""
    N = n ** d
    rows, cols, vals = [np.arange(N)], [np.arange(N)], [np.full(N, 2.0 * d)]
    for p, q, _ in _grid_shift_pairs(n, d):
        rows += [p, q]
        cols += [q, p]
        vals += [np.full(p.size, -1.0), np.full(p.size, -1.0)]
    A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    return _to_csc(A)


def gaussian_random_field(n: int, d: int, corr_len: float, variance: float, seed: int) -> np.ndarray:
    """Stationary Gaussian field on the n^d grid, squared-exponential covariance.

    C(r) = variance * exp(-r^2 / (2 corr_len^2)) (r in grid cells), sampled by
    circulant embedding on a periodic (2n)^d grid: g = Re IFFT(sqrt(FFT(C)) *
    FFT(xi)), xi ~ N(0,1) from ``numpy.random.default_rng(seed)``, restricted to
    the first n^d block and standardised to sample mean 0 / variance ``variance``.
    """
    M = 2 * n
    ax = np.minimum(np.arange(M), M - np.arange(M)).astype(np.float64)
    r2 = np.zeros((M,) * d)
    for k in range(d):
        shape = [1] * d
        shape[k] = M
        r2 = r2 + (ax.reshape(shape) ** 2)
    C = np.exp(-r2 / (2.0 * corr_len ** 2))
    S = np.maximum(np.fft.fftn(C).real, 0.0)
    rng = np.random.default_rng(seed)
    xi = rng.standard_normal((M,) * d)
    g = np.fft.ifftn(np.sqrt(S) * np.fft.fftn(xi)).real
    g = g[(slice(0, n),) * d]
    g = (g - g.mean()) / g.std()
    return (np.sqrt(variance) * g).ravel()


def diffusion(k: np.ndarray, n: int, d: int):
    """-div(k grad u) with harmonic-mean face coefficients (cell-centred, Dirichlet).

    Face coefficient between cells p and q: 2 k_p k_q / (k_p + k_q); a face to the
    boundary uses k_p.  Diagonal = sum of the cell's face coefficients.
    """
    N = n ** d
    k = np.asarray(k, dtype=np.float64).ravel()
    diag = np.zeros(N)
    rows, cols, vals = [], [], []
    idx = np.arange(N).reshape((n,) * d)
    for ax in range(d):
        # every cell has 2 faces along ax; interior faces are shared
        for p, q, a in _grid_shift_pairs(n, d):
            if a != ax:
                continue
            kf = 2.0 * k[p] * k[q] / (k[p] + k[q])
            np.add.at(diag, p, kf)
            np.add.at(diag, q, kf)
            rows += [p, q]
            cols += [q, p]
            vals += [-kf, -kf]
        lo = [slice(None)] * d
        hi = [slice(None)] * d
        lo[ax] = 0
        hi[ax] = n - 1
        for b in (idx[tuple(lo)].ravel(), idx[tuple(hi)].ravel()):
            np.add.at(diag, b, k[b])
    rows.append(np.arange(N))
    cols.append(np.arange(N))
    vals.append(diag)
    A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    return _to_csc(A)


def diffusion_lognormal(n: int, d: int = 3, seed: int = 2, corr_len: float = 8.0, variance: float = 1.0):
    """k = exp(g), g a Gaussian random field (variable-coefficient diffusion workload)."""
    g = gaussian_random_field(n, d, corr_len, variance, seed)
    return diffusion(np.exp(g), n, d)


def diffusion_binary(n: int, d: int = 3, seed: int = 3, corr_len: float = 8.0, contrast_exp: float = 3.0):
    """High-contrast channels: k = 10^(contrast_exp * sign(g))."""
    g = gaussian_random_field(n, d, corr_len, 1.0, seed)
    return diffusion(10.0 ** (contrast_exp * np.sign(g)), n, d)


def convection_diffusion_2d(n: int, eps: float = 1e-2):
    """-eps Lap u + w.grad u on the unit square, first-order upwinding.

    w is a unit-magnitude rotating vortex about (0.5, 0.5):
    w = (-(y-0.5), x-0.5) / |(x-0.5, y-0.5)| (w = 0 at the centre point).
    Grid spacing h = 1/(n+1); unknown (i, j) sits at (x, y) = ((i+1)h, (j+1)h).
    """
    h = 1.0 / (n + 1)
    N = n * n
    ii, jj = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    x = (ii.ravel() + 1) * h - 0.5
    y = (jj.ravel() + 1) * h - 0.5
    r = np.hypot(x, y)
    with np.errstate(invalid="ignore", divide="ignore"):
        wx = np.where(r > 0, -y / r, 0.0)
        wy = np.where(r > 0, x / r, 0.0)
    idx = np.arange(N).reshape(n, n)
    diag = np.full(N, 4.0 * eps / h ** 2) + (np.abs(wx) + np.abs(wy)) / h
    rows, cols, vals = [np.arange(N)], [np.arange(N)], [diag]
    # axis 0 couples (i,j)-(i+1,j) through wx; axis 1 through wy
    for ax, w in ((0, wx), (1, wy)):
        lo = [slice(None)] * 2
        hi = [slice(None)] * 2
        lo[ax] = slice(0, n - 1)
        hi[ax] = slice(1, n)
        p = idx[tuple(lo)].ravel()
        q = idx[tuple(hi)].ravel()
        # row p, neighbour q (q is the "+" neighbour of p): diffusion -eps/h^2,
        # upwind uses q when w_p < 0: +w_p/h * (u_q) ... i.e. coefficient min(w_p,0)/h
        rows += [p, q]
        cols += [q, p]
        vals += [-eps / h ** 2 + np.minimum(w[p], 0.0) / h, -eps / h ** 2 - np.maximum(w[q], 0.0) / h]
    A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    return _to_csc(A)


def rhs_normal(n: int, seed: int, nrhs: int = 1) -> np.ndarray:
    """b ~ N(0,1) from numpy.random.default_rng(seed); shape (n,) or (n, nrhs)."""
    rng = np.random.default_rng(seed)
    if nrhs == 1:
        return rng.standard_normal(n)
    return np.asfortranarray(rng.standard_normal((nrhs, n)).T)


WORKLOADS = {
    # name: (builder, grid n, dim, nlevels, tol, rhs seed)
    "lapl2d_64": (lambda: laplacian(64, 2), 64, 2, 6, 1e-2, 0),
    "lapl3d_64": (lambda: laplacian(64, 3), 64, 3, 12, 1e-2, 1),
    "diff3d_64": (lambda: diffusion_lognormal(64, 3, seed=2), 64, 3, 12, 1e-2, 2),
    "chan3d_64": (lambda: diffusion_binary(64, 3, seed=3), 64, 3, 12, 1e-2, 3),
    "convdiff2d_1024": (lambda: convection_diffusion_2d(1024), 1024, 2, 14, 1e-2, 4),
}
