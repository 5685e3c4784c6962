"""Seeded synthetic sparse systems (CSR, int32 indices, sorted columns, diagonal
present) for the stencil problems the solve path is measured on.

The reference ships no matrices or generators (its drivers read Matrix Market
files, hip/main_solve_base.cpp:25-120); these stand in for them.  All operators
are assembled h^2-scaled so that the diagonal stays O(1)-O(100), which keeps
BF16/FP16 factor storage in range.

  poisson2d_5pt(nx)          4 / -1, Dirichlet, n = nx^2
  poisson3d_7pt(nx)          6 / -1, Dirichlet, n = nx^3
  convdiff3d_27pt(nx, pe)    diffusion 26 / -1 over the 26 neighbours, plus
                             first-order upwind convection on the 6 face
                             neighbours with velocity pe * (1, 0.5, 0.25):
                             a_ii += c_d, a_{i, i - e_d} -= c_d (nonsymmetric)
  varcoef3d_7pt(nx, seed)    k = exp(g), g ~ N(0,1) per cell; face coefficient
                             = harmonic mean of the two cells; a boundary face
                             uses the cell's own k; SPD.
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "poisson2d_5pt",
    "poisson3d_7pt",
    "convdiff3d_27pt",
    "varcoef3d_7pt",
    "rhs_uniform",
    "CSRMatrix",
]


class CSRMatrix:
    """Plain host CSR container (0-based, int32 indices, float64 values)."""

    def __init__(self, n, rowptr, colidx, val, name=""):
        self.n = int(n)
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self.colidx = np.ascontiguousarray(colidx, dtype=np.int32)
        self.val = np.ascontiguousarray(val, dtype=np.float64)
        self.name = name

    @property
    def nnz(self):
        return int(self.rowptr[-1] - self.rowptr[0])  # rowptr[0] is the index base (0 or 1)

    def to_scipy(self):
        import scipy.sparse as sp

        return sp.csr_matrix((self.val, self.colidx, self.rowptr), shape=(self.n, self.n))

    def __repr__(self):
        return f"CSRMatrix({self.name!r}, n={self.n}, nnz={self.nnz})"


def _assemble(shape, offsets, coef):
    """Build CSR from a structured stencil.

    shape   grid shape (z, y, x) or (y, x); row index is C-order (x fastest)
    offsets list of integer offset tuples, sorted so column indices increase
    coef    array (n, len(offsets)) of coefficients for every cell and offset
    """
    dims = len(shape)
    n = int(np.prod(shape))
    idx = np.arange(n, dtype=np.int64).reshape(shape)
    cols = np.empty((n, len(offsets)), dtype=np.int64)
    mask = np.empty((n, len(offsets)), dtype=bool)
    grids = np.indices(shape)
    for t, off in enumerate(offsets):
        ok = np.ones(shape, dtype=bool)
        for d in range(dims):
            g = grids[d] + off[d]
            ok &= (g >= 0) & (g < shape[d])
        mask[:, t] = ok.reshape(-1)
        lin = 0
        stride = 1
        for d in reversed(range(dims)):
            lin = lin + off[d] * stride
            stride *= shape[d]
        cols[:, t] = idx.reshape(-1) + lin
    del grids
    counts = mask.sum(axis=1)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rowptr[1:])
    colidx = cols[mask].astype(np.int32)
    val = coef[mask].astype(np.float64)
    return n, rowptr.astype(np.int32), colidx, val


def _sorted_offsets(dims, full):
    rng = (-1, 0, 1)
    if dims == 2:
        offs = [(dy, dx) for dy in rng for dx in rng]
    else:
        offs = [(dz, dy, dx) for dz in rng for dy in rng for dx in rng]
    if not full:
        offs = [o for o in offs if sum(abs(c) for c in o) <= 1]
    return offs  # lexicographic order == increasing column index


def poisson2d_5pt(nx: int) -> CSRMatrix:
    offs = _sorted_offsets(2, full=False)
    n = nx * nx
    coef = np.empty((n, len(offs)))
    for t, o in enumerate(offs):
        coef[:, t] = 4.0 if o == (0, 0) else -1.0
    nn, rp, ci, v = _assemble((nx, nx), offs, coef)
    return CSRMatrix(nn, rp, ci, v, f"poisson2d_5pt_{nx}")


def poisson3d_7pt(nx: int) -> CSRMatrix:
    offs = _sorted_offsets(3, full=False)
    n = nx ** 3
    coef = np.empty((n, len(offs)))
    for t, o in enumerate(offs):
        coef[:, t] = 6.0 if o == (0, 0, 0) else -1.0
    nn, rp, ci, v = _assemble((nx, nx, nx), offs, coef)
    return CSRMatrix(nn, rp, ci, v, f"poisson3d_7pt_{nx}")


def convdiff3d_27pt(nx: int, pe: float = 50.0, velocity=(1.0, 0.5, 0.25)) -> CSRMatrix:
    """27-point diffusion (26 / -1) + first-order upwind convection.

    velocity is (vx, vy, vz); each component is multiplied by pe.  With all
    components positive the upwind neighbour is the one at -e_d.
    """
    offs = _sorted_offsets(3, full=True)
    n = nx ** 3
    coef = np.empty((n, len(offs)), dtype=np.float64)
    vx, vy, vz = (pe * velocity[0], pe * velocity[1], pe * velocity[2])
    conv = {(0, 0, -1): vx, (0, -1, 0): vy, (-1, 0, 0): vz}
    diag = 26.0 + abs(vx) + abs(vy) + abs(vz)
    for t, o in enumerate(offs):
        if o == (0, 0, 0):
            coef[:, t] = diag
        else:
            coef[:, t] = -1.0 - conv.get(o, 0.0)
    nn, rp, ci, v = _assemble((nx, nx, nx), offs, coef)
    return CSRMatrix(nn, rp, ci, v, f"convdiff3d_27pt_{nx}_pe{pe:g}")


def varcoef3d_7pt(nx: int, seed: int = 0) -> CSRMatrix:
    rng = np.random.default_rng(seed)
    k = np.exp(rng.standard_normal((nx, nx, nx)))
    n = nx ** 3
    offs = _sorted_offsets(3, full=False)
    coef = np.zeros((n, len(offs)), dtype=np.float64)
    diag = np.zeros((nx, nx, nx))
    center = offs.index((0, 0, 0))
    for t, o in enumerate(offs):
        if o == (0, 0, 0):
            continue
        # neighbour coefficient with edge replication for the boundary face
        kn = np.pad(k, 1, mode="edge")[
            1 + o[0]: 1 + o[0] + nx, 1 + o[1]: 1 + o[1] + nx, 1 + o[2]: 1 + o[2] + nx
        ]
        face = 2.0 * k * kn / (k + kn)
        diag += face  # boundary faces (Dirichlet) also contribute to the diagonal
        coef[:, t] = -face.reshape(-1)
    coef[:, center] = diag.reshape(-1)
    nn, rp, ci, v = _assemble((nx, nx, nx), offs, coef)
    return CSRMatrix(nn, rp, ci, v, f"varcoef3d_7pt_{nx}_s{seed}")


def rhs_uniform(n: int, seed: int = 0, low: float = -1.0, high: float = 1.0) -> np.ndarray:
    """b ~ U(low, high) from numpy's PCG64 generator with the given seed."""
    return np.random.default_rng(seed).uniform(low, high, n)
