"""Oracle (test infrastructure only): the exact solution of the reference's
pressure operator on a uniform periodic block mesh, by FFT.

On a uniform periodic mesh every vertex patch is conforming, so the inverse
face metric is diagonal, K_ff = 1 / (|f| d_f) (`_local_inverse_metric` on a
conforming patch, src/operators/gradient.jl:275-292 of
ronaldremmerswaal/TwoPhaseAMR.jl), and the factorized action with kappa = 1
(`FactorizedEllipticOperator` mul!, src/operators/elliptic.jl:1125-1180) is
the integrated five-point operator (A x)_c = sum over the four neighbours n of
(|f| / d_f) (x_c - x_n), with |f| / d_f = h_y / h_x across x faces and
h_x / h_y across y faces.  The discrete Fourier transform diagonalises it, so
`solve!` (src/solvers/multigrid/elliptic_solver.jl:628-675: b = V f, the RHS
volume mean removed, the solution volume mean removed) has the exact answer
computed here, to be compared with an iterative solve of the same system.

Cell order is the reference's: blocks sorted by (level, j, i), so on a uniform
level-0 mesh block (bi, bj) is number bj * nbx + bi, and cell (i, j) of a
block is number j * nx + i inside it (src/mesh/topology/mesh.jl:28-30).
"""
from __future__ import annotations

import numpy as np


def to_grid(v, base_mesh, block_size):
    """Cell-order vector -> (ny_total, nx_total) array."""
    (NX, NY), (bx, by) = base_mesh, block_size
    nbx, nby = NX // bx, NY // by
    return np.asarray(v).reshape(nby, nbx, by, bx).transpose(0, 2, 1, 3).reshape(NY, NX)


def from_grid(g, base_mesh, block_size):
    (NX, NY), (bx, by) = base_mesh, block_size
    nbx, nby = NX // bx, NY // by
    return np.ascontiguousarray(np.asarray(g).reshape(nby, by, nbx, bx).transpose(0, 2, 1, 3)).reshape(-1)


def apply(x, base_mesh, block_size, extent=(1.0, 1.0)):
    """The integrated operator A x on the uniform periodic mesh."""
    hx, hy = extent[0] / base_mesh[0], extent[1] / base_mesh[1]
    g = to_grid(x, base_mesh, block_size)
    cx, cy = hy / hx, hx / hy
    y = cx * (2 * g - np.roll(g, 1, axis=1) - np.roll(g, -1, axis=1)) + \
        cy * (2 * g - np.roll(g, 1, axis=0) - np.roll(g, -1, axis=0))
    return from_grid(y, base_mesh, block_size)


def solve(rhs_strong, base_mesh, block_size, extent=(1.0, 1.0)):
    """`solve!` of A x = V f (mean-free) to machine precision: returns x with
    zero volume mean."""
    NX, NY = base_mesh
    hx, hy = extent[0] / NX, extent[1] / NY
    b = to_grid(np.asarray(rhs_strong, dtype=np.float64) * (hx * hy), base_mesh, block_size)
    b = b - b.mean()
    kx = 2 * np.pi * np.fft.rfftfreq(NX)
    ky = 2 * np.pi * np.fft.fftfreq(NY)
    lam = (hy / hx) * (2 - 2 * np.cos(kx))[None, :] + (hx / hy) * (2 - 2 * np.cos(ky))[:, None]
    bh = np.fft.rfft2(b)
    lam[0, 0] = 1.0
    xh = bh / lam
    xh[0, 0] = 0.0
    x = np.fft.irfft2(xh, s=(NY, NX))
    return from_grid(x - x.mean(), base_mesh, block_size)
