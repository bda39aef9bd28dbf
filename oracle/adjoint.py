"""Oracle (test infrastructure only): CPU adjoint of TwoPhaseAMR.jl's pressure
solve, for checking the B200 gradient kernels.

The forward map is `solve!(p, solver, f)` with compatibility :project
(src/solvers/multigrid/elliptic_solver.jl:628-675 of
ronaldremmerswaal/TwoPhaseAMR.jl):

    b = V f,  b <- Pi b = b - V (1'b)/(1'V)        (_project_component_rhs!, :153-190)
    S(kappa) x = b,  S = J' sqrt(k) K sqrt(k) J    (elliptic.jl:157-257)
    p = G x = x - 1 (V'x)/(1'V)                    (_remove_component_volume_means!, :132-151)

The reference differentiates nothing; this module restates the adjoint of that
map.  S is symmetric and Pi' = G, so for a loss J with dJ/dp = pbar the adjoint
state is lam = G S^+ Pi pbar (the same solve with strong right-hand side
pbar / V) and

    dJ/df     = V lam
    dJ/dkappa = -lam' (dS/dkappa_f) p = -[w (K sqrt(k) u) + u (K sqrt(k) w)] / (2 sqrt(k))

with u = J p and w = J lam.  Only the single-component case (one connected
domain, no gauged components) is restated; every configuration here has it.
`exact_solve` solves the gauged system directly (sparse LU of the bordered
matrix), so finite differences of the loss carry no Krylov error.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .krylov import solve as krylov_solve


def exact_solve(op, rhs_strong):
    """p = G S^+ Pi (V f) by a direct solve of [S 1; V' 0][p; mu] = [Pi V f; 0]."""
    v = op.volumes
    n = len(v)
    b = np.asarray(rhs_strong, dtype=np.float64) * v
    b = b - v * np.sum(b) / np.sum(v)
    ones = np.ones((n, 1))
    M = sp.bmat([[op.matrix, sp.csr_matrix(ones)], [sp.csr_matrix(v[None, :]), None]], format="csc")
    sol = spla.spsolve(M, np.concatenate([b, [0.0]]))
    return sol[:n]


def face_gradient(op, p, lam):
    """-lam' (dS/dkappa_f) p for every interior face (needs kappa > 0 on faces
    with off-diagonal K entries)."""
    u = op.J @ p
    w = op.J @ lam
    sk = op.sqrt_kappa
    d = op.K.diagonal()
    off = (op.K - sp.diags(d)).tocsr()
    U = off @ (sk * u)
    W = off @ (sk * w)
    g = 2.0 * d * u * w
    nz = (U != 0) | (W != 0)
    g[nz] += (w[nz] * U[nz] + u[nz] * W[nz]) / sk[nz]
    return -0.5 * g


def adjoint(op, p, pbar, mg=None, *, rtol=1e-12, exact=False):
    """(rhs_bar, kappa_bar, lam) for the cotangent pbar of the solution p.  The
    adjoint system is solved by the oracle's CG + V-cycle (the reference's CPU
    solve), or directly when `exact`."""
    v = op.volumes
    strong = np.asarray(pbar, dtype=np.float64) / v
    if exact:
        lam = exact_solve(op, strong)
    else:
        lam, stats = krylov_solve(op, mg, strong, rtol=rtol)
        if not stats.converged:
            raise RuntimeError("oracle adjoint solve did not converge")
    return v * lam, face_gradient(op, p, lam), lam


# ---- the C5 loss: J = 1/2 ||p - p_t||^2 over fine cells near the centre ----

def loss_mask(centers, center=(0.5, 0.6), radius=0.2, volumes=None, finest_volume=None):
    """Cells of the finest level whose centre lies within `radius` of `center`."""
    x, y = centers
    mask = np.hypot(x - center[0], y - center[1]) < radius
    if volumes is not None and finest_volume is not None:
        mask &= np.isclose(volumes, finest_volume, rtol=1e-12, atol=0.0)
    return mask


def loss(p, target, mask):
    d = np.where(mask, p - target, 0.0)
    return 0.5 * float(np.dot(d, d))


def loss_cotangent(p, target, mask):
    return np.where(mask, p - target, 0.0)
