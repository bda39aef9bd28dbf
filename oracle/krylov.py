"""Oracle (test infrastructure only): CPU restatement of the Krylov wrapper of
TwoPhaseAMR.jl's pressure solve.

Reference (ronaldremmerswaal/TwoPhaseAMR.jl):
  src/solvers/multigrid/elliptic_solver.jl:369-378  `StrongResidualCallback`
  src/solvers/multigrid/elliptic_solver.jl:403-464  `_run_krylov!` (atol=rtol=0, callback)
  src/solvers/multigrid/elliptic_solver.jl:467-485  `_guarded_roundoff_target!`
  src/solvers/multigrid/elliptic_solver.jl:487-526  `_run_krylov_reliably!` (restarts)
  src/solvers/multigrid/elliptic_solver.jl:550-612  `_solve_krylov_with_stats!`
  src/solvers/multigrid/elliptic_solver.jl:628-675  `solve!` (prepare: b *= V, projection)
  src/solvers/multigrid/cycles.jl:108-260           roundoff floor, residual norms
  src/solvers/multigrid/stats.jl:15-30              `LinearSolverStats`

The CG recurrence is Krylov.jl 0.10's `cg!` (Project.toml compat "0.10";
Krylov.jl is not vendored with the reference), restated from its published
algorithm: warm start through `dx`, `z = M \\ r`, `gamma = r'z`,
`alpha = gamma / p'Ap`, zero-curvature guard `p'Ap <= eps * pNorm^2`,
machine stop `sqrt(gamma) + 1 <= 1`, `beta = gamma_next / gamma`, and the user
callback after every iteration.  The bits of its dot products are not pinned.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .operator import project_component_rhs, remove_component_volume_means

EPS = np.finfo(np.float64).eps


def strong_max(r, volumes):
    """`_strong_residual_maximum` (cycles.jl:230-260)."""
    sel = volumes > 0
    return float(np.max(np.abs(r[sel]) / volumes[sel])) if np.any(sel) else 0.0


def integrated_norms(r, volumes):
    """`_integrated_residual_norms` (cycles.jl:210-221)."""
    sel = volumes > 0
    strong = r[sel] / volumes[sel]
    return float(np.sqrt(np.sum(volumes[sel] * strong ** 2) / np.sum(volumes[sel]))), strong_max(r, volumes)


def roundoff_floor(op, x, b, volumes):
    """`_roundoff_residual_floor!` for the factorized action (cycles.jl:108-206)."""
    bound = op.abs_apply(x)
    sel = volumes > 0
    scale = 0.0
    if np.any(sel):
        scale = max(float(np.max(bound[sel] / volumes[sel])), float(np.max(np.abs(b[sel]) / volumes[sel])))
    return 128 * EPS * max(1.0, scale)


@dataclass
class CGResult:
    x: np.ndarray
    niter: int
    status: str


def cg(apply, b, x0, M, target, volumes, itmax):
    """Krylov.jl 0.10 `cg!` with `M` (ldiv), atol = rtol = 0 and the strong
    residual callback of `_run_krylov!`."""
    n = len(b)
    dx = x0.copy()
    x = np.zeros(n)
    r = b - apply(dx)
    z = M(r)
    p = z.copy()
    gamma = float(r @ z)
    if gamma == 0:
        return CGResult(x + dx, 0, "zero residual")
    it = 0
    pnorm2 = gamma
    eps_stop = 0.0
    rnorm = np.sqrt(gamma)
    solved = rnorm <= eps_stop
    tired = it >= itmax
    zero_curv = False
    user_exit = False
    while not (solved or tired or zero_curv or user_exit):
        Ap = apply(p)
        pAp = float(p @ Ap)
        if pAp <= EPS * pnorm2 and abs(pAp) <= EPS * pnorm2:
            zero_curv = True
            continue
        alpha = gamma / pAp
        x += alpha * p
        r -= alpha * Ap
        z = M(r)
        gamma_next = float(r @ z)
        rnorm = np.sqrt(gamma_next) if gamma_next >= 0 else np.nan
        solved = (rnorm + 1.0 <= 1.0) or (rnorm <= eps_stop)
        if not solved:
            beta = gamma_next / gamma
            pnorm2 = gamma_next + beta ** 2 * pnorm2
            gamma = gamma_next
            p = z + beta * p
        it += 1
        tired = it >= itmax
        user_exit = strong_max(r, volumes) <= target
    return CGResult(x + dx, it, "zero curvature" if zero_curv else "done")


@dataclass
class LinearSolverStats:
    """`LinearSolverStats` (stats.jl:15-30)."""

    cycles: int = 0
    converged: bool = False
    compatible: bool = True
    initial_l2: float = np.inf
    initial_linf: float = np.inf
    final_l2: float = np.inf
    final_linf: float = np.inf
    target_linf: float = np.inf
    residual_scale: float = 1.0
    removed_rhs_mean: float = 0.0
    removed_rhs_component_means: list = field(default_factory=list)
    removed_rhs_component_anchors: list = field(default_factory=list)
    method: str = "cg"
    preconditioner: str = "tree_geometric_multigrid"


def guarded_target(op, x, b, volumes, target, initial_linf, current_linf):
    """`_guarded_roundoff_target!` (elliptic_solver.jl:467-485)."""
    if not (np.isfinite(initial_linf) and np.isfinite(current_linf) and target < current_linf < initial_linf):
        return target
    floor = roundoff_floor(op, x, b, volumes)
    return max(target, floor) if np.isfinite(floor) and floor < initial_linf / 100 else target


def solve(op, mg, rhs_strong, x0=None, *, rtol=1e-10, atol=0.0, max_cycles=100,
          compatibility="project", preconditioner=True):
    """`solve!(solution, solver, rhs)` (elliptic_solver.jl:628-675).  `rhs_strong`
    is the strong-form right-hand side in cell order; returns (x, stats)."""
    if not 0 <= rtol < 1:
        raise ValueError("rtol must lie in [0, 1)")
    if atol < 0:
        raise ValueError("atol must be nonnegative")
    if max_cycles < 0:
        raise ValueError("max_cycles must be nonnegative")
    if compatibility not in ("project", "error"):
        raise ValueError("compatibility must be :project or :error")
    volumes = op.volumes
    comp = op.components
    stats = LinearSolverStats()
    x = np.zeros(op.mesh.ncells) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    b = np.asarray(rhs_strong, dtype=np.float64) * volumes
    b[volumes == 0] = 0.0
    x[volumes == 0] = 0.0
    removed = 0.0
    if op.singular:
        if compatibility == "error":
            for s in range(len(comp["anchors"])):
                sel = comp["slots"] == s
                tol = 256 * EPS * max(1.0, float(np.sum(np.abs(b[sel]))))
                if abs(float(np.sum(b[sel]))) > tol:
                    raise ValueError("Poisson right-hand side has nonzero volume mean")
        b, means, removed = project_component_rhs(b, volumes, comp)
        stats.removed_rhs_component_means = list(means)
        stats.removed_rhs_component_anchors = [int(a) + 1 for a in comp["anchors"]]
        x = remove_component_volume_means(x, volumes, comp)
    r = b - op.apply(x)
    initial_l2, initial_linf = integrated_norms(r, volumes)
    floor = roundoff_floor(op, x, b, volumes)
    target = max(atol, rtol * max(initial_linf, EPS), floor)
    M = mg.ldiv if (preconditioner and mg is not None) else (lambda v: v.copy())
    total = 0
    if initial_linf > target:
        while total < max_cycles:
            res = cg(op.apply, b, x, M, target, volumes, max_cycles - total)
            total += res.niter
            x = res.x
            if op.singular:
                x = remove_component_volume_means(x, volumes, comp)
            r = b - op.apply(x)
            final_linf = strong_max(r, volumes)
            eff = guarded_target(op, x, b, volumes, target, initial_linf, final_linf)
            if final_linf <= eff:
                break
            if not np.isfinite(final_linf) or res.niter == 0:
                break
    if op.singular:
        x = remove_component_volume_means(x, volumes, comp)
    r = b - op.apply(x)
    final_l2, final_linf = integrated_norms(r, volumes)
    target = guarded_target(op, x, b, volumes, target, initial_linf, final_linf)
    stats.cycles = total
    stats.converged = bool(np.isfinite(final_linf) and np.isfinite(target) and final_linf <= target)
    stats.initial_l2, stats.initial_linf = initial_l2, initial_linf
    stats.final_l2, stats.final_linf = final_l2, final_linf
    stats.target_linf = target
    stats.residual_scale = max(initial_linf, EPS)
    stats.removed_rhs_mean = removed
    if mg is None or not preconditioner:
        stats.preconditioner = "none"
    return x, stats
