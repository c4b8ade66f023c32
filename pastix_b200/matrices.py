"""Synthetic sparse matrices of the benchmark workloads, generated directly as CSC.

Grid vertex (i, j, k) of an nx*ny*nz grid is numbered ``i + nx*j + nx*ny*k``, the
numbering ``pastixOrderGrid`` assumes (order/order_grids.c:166).  spm's own Laplacian
generators put ``degree*alpha`` on the diagonal and scaled off-diagonals
(spm/src/z_spm_laplacian.c:146,268), which are not the matrices wanted here, so the
values are built in numpy instead.

Symmetric matrices are returned as their lower triangle (SpmSymmetric CSC); general
matrices as the full pattern (SpmGeneral CSC).  Row indices are sorted per column.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class CSC:
    n: int
    colptr: np.ndarray  # int64 [n+1]
    rowind: np.ndarray  # int64 [nnz]
    values: np.ndarray  # float64 [nnz]
    symmetric: bool     # True: lower triangle of a symmetric matrix
    grid: tuple         # (nx, ny, nz) for the grid nested-dissection ordering
    name: str = ""

    @property
    def nnz(self) -> int:
        return int(self.colptr[-1])

    def to_dense(self) -> np.ndarray:
        a = np.zeros((self.n, self.n))
        cols = np.repeat(np.arange(self.n), np.diff(self.colptr))
        a[self.rowind, cols] = self.values
        if self.symmetric:
            a = a + np.tril(a, -1).T
        return a

    def full(self) -> "CSC":
        """Both triangles (for a symmetric matrix), as a general CSC."""
        if not self.symmetric:
            return self
        cols = np.repeat(np.arange(self.n), np.diff(self.colptr))
        off = self.rowind != cols
        r = np.concatenate([self.rowind, cols[off]])
        c = np.concatenate([cols, self.rowind[off]])
        v = np.concatenate([self.values, self.values[off]])
        return _coo_to_csc(self.n, r, c, v, False, self.grid, self.name)

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """y = A x for x of shape (n,) or (n, nrhs), float64."""
        x2 = x.reshape(self.n, -1)
        cols = np.repeat(np.arange(self.n), np.diff(self.colptr))
        y = np.zeros_like(x2, dtype=np.float64)
        np.add.at(y, self.rowind, self.values[:, None] * x2[cols])
        if self.symmetric:
            off = self.rowind != cols
            np.add.at(y, cols[off], self.values[off, None] * x2[self.rowind[off]])
        return y.reshape(x.shape)

    def norm_fro(self) -> float:
        if self.symmetric:
            cols = np.repeat(np.arange(self.n), np.diff(self.colptr))
            off = self.rowind != cols
            return float(np.sqrt(np.sum(self.values ** 2) + np.sum(self.values[off] ** 2)))
        return float(np.linalg.norm(self.values))

    def norm_one(self) -> float:
        f = self.full()
        cols = np.repeat(np.arange(f.n), np.diff(f.colptr))
        return float(np.max(np.bincount(cols, np.abs(f.values), minlength=f.n)))


def _coo_to_csc(n, r, c, v, symmetric, grid, name) -> CSC:
    order = np.lexsort((r, c))
    r, c, v = r[order], c[order], v[order]
    colptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(colptr, c + 1, 1)
    colptr = np.cumsum(colptr)
    return CSC(n, colptr, r.astype(np.int64), v.astype(np.float64), symmetric, grid, name)


def _stencil_offsets(points: int, dims: int):
    if dims == 2:
        if points != 5:
            raise ValueError("2D stencils: 5 points")
        return [(1, 0, 0), (0, 1, 0)]
    if points == 7:
        return [(1, 0, 0), (0, 1, 0), (0, 0, 1)]
    if points == 27:
        offs = []
        for dk in (-1, 0, 1):
            for dj in (-1, 0, 1):
                for di in (-1, 0, 1):
                    d = (di, dj, dk)
                    # keep one of each (d, -d) pair: the one that points to a larger index
                    lin = di + 3 * dj + 9 * dk
                    if lin > 0:
                        offs.append(d)
        return offs
    raise ValueError("3D stencils: 7 or 27 points")


def _grid_pairs(nx, ny, nz, offsets):
    """(lo, hi) vertex pairs for each stencil offset pointing to the larger index."""
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    lo_all, hi_all, dir_all = [], [], []
    for oi, (di, dj, dk) in enumerate(offsets):
        ii, jj, kk = i + di, j + dj, k + dk
        ok = (ii >= 0) & (ii < nx) & (jj >= 0) & (jj < ny) & (kk >= 0) & (kk < nz)
        lo = (i + nx * j + nx * ny * k)[ok]
        hi = (ii + nx * jj + nx * ny * kk)[ok]
        lo_all.append(lo)
        hi_all.append(hi)
        dir_all.append(np.full(lo.shape, oi))
    return np.concatenate(lo_all), np.concatenate(hi_all), np.concatenate(dir_all)


def laplacian(nx: int, ny: int, nz: int = 1, points: int = 7, diag: float | None = None,
              off: float = -1.0, shift: float = 0.0) -> CSC:
    """Constant-coefficient Laplacian: ``diag + shift`` on the diagonal, ``off`` elsewhere.

    ``diag`` defaults to the stencil's neighbour count (6 for 7-pt, 26 for 27-pt,
    4 for the 2D 5-pt).  Lower-triangle symmetric CSC.
    """
    dims = 2 if nz == 1 and points == 5 else 3
    offsets = _stencil_offsets(points, dims)
    if diag is None:
        diag = float(points - 1)
    n = nx * ny * nz
    lo, hi, _ = _grid_pairs(nx, ny, nz, offsets)
    r = np.concatenate([np.arange(n), hi])
    c = np.concatenate([np.arange(n), lo])
    v = np.concatenate([np.full(n, diag + shift), np.full(lo.shape, off)])
    return _coo_to_csc(n, r, c, v, True, (nx, ny, nz), f"lap{points}_{nx}x{ny}x{nz}")


def convection_diffusion(nx: int, ny: int, nz: int, seed: int = 0, vmax: float = 50.0) -> CSC:
    """Upwind 7-point convection-diffusion on the unit cube, scaled by h^2.

    -Δu + v·∇u with diffusion 1 and per-cell velocity components drawn uniform
    [0, vmax] from ``seed``; h = 1/(n+1).  Backward (upwind) differences for the
    convection term give, per cell c and axis d:
        A[c, c]       += 2 + v_d h
        A[c, c - e_d]  = -1 - v_d h
        A[c, c + e_d]  = -1
    Nonsymmetric values on a symmetric pattern (general CSC, full pattern).
    """
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    h = 1.0 / (max(nx, ny, nz) + 1)
    vel = rng.uniform(0.0, vmax, size=(3, n))
    offsets = _stencil_offsets(7, 3)
    lo, hi, d = _grid_pairs(nx, ny, nz, offsets)
    # entry (row=hi, col=lo): row hi's backward neighbour is lo -> -1 - v_d(hi) h
    # entry (row=lo, col=hi): row lo's forward neighbour is hi  -> -1
    diagv = 6.0 + h * vel.sum(axis=0)
    r = np.concatenate([np.arange(n), hi, lo])
    c = np.concatenate([np.arange(n), lo, hi])
    v = np.concatenate([diagv, -1.0 - vel[d, hi] * h, np.full(lo.shape, -1.0)])
    return _coo_to_csc(n, r, c, v, False, (nx, ny, nz), f"convdiff_{nx}x{ny}x{nz}")


def lambda_max_5pt(side: int) -> float:
    """Largest eigenvalue of the 2D 5-point Dirichlet Laplacian (4 on the diagonal)."""
    return 4.0 + 4.0 * np.cos(np.pi / (side + 1))


def shifted_laplacian_2d(side: int, sigma: float) -> CSC:
    """2D 5-point Laplacian minus sigma*I (symmetric indefinite for sigma > lambda_min)."""
    return laplacian(side, side, 1, points=5, diag=4.0, shift=-sigma)


def rhs_from_xtrue(A: CSC, nrhs: int, seed: int):
    """x_true i.i.d. uniform[-1, 1] from ``seed`` and b = A x_true (column-major n x nrhs)."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1.0, 1.0, size=(A.n, nrhs))
    b = A.matvec(x)
    return np.asfortranarray(x), np.asfortranarray(b)


def indefinite_batch(nsys: int = 4096, seed: int = 2024, side_min: int = 16, side_max: int = 128):
    """The batched indefinite workload: nsys 2D 5-point Laplacians with grid sides
    log-uniform in [side_min, side_max] (n = 256 .. 16,384 at the defaults), each
    shifted by -sigma I with sigma uniform in (0, 0.5 lambda_max).  Returns the sides
    and shifts (the matrices are ``shifted_laplacian_2d(side, sigma)``)."""
    rng = np.random.default_rng(seed)
    sides = np.floor(np.exp(rng.uniform(np.log(side_min), np.log(side_max + 1), nsys))).astype(int)
    sides = sides.clip(side_min, side_max)
    sig = rng.uniform(0.0, 0.5, nsys) * np.array([lambda_max_5pt(int(s)) for s in sides])
    return sides, sig
