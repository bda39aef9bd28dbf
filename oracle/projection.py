"""Oracle (test infrastructure only): CPU restatement of TwoPhaseAMR.jl's
one-velocity projection step around the pressure solve and of the two-phase
coefficients and surface-tension force that feed it.

Reference (ronaldremmerswaal/TwoPhaseAMR.jl):
  src/interface/interface_field.jl:248-291   `_refresh_conditional_fraction!`
                                             (no embedded geometry: open = 1)
  src/two_phase/forces.jl:23-36, 69-84       `_staggered_liquid_fraction`,
                                             `_mixture_density!`
  src/two_phase/forces.jl:113-140            `PoissonOperator(field; density)`:
                                             kappa = inv.(rho)
  src/two_phase/forces.jl:312-314, 345-378   CSF / CGFM jumps, `_surface_tension_jumps!`
                                             (constant curvature)
  src/two_phase/forces.jl:179-209            `_weighted_jump_force!`
  src/operators/gradient.jl:433-441          `_pressure_jump!`
  src/operators/elliptic.jl:1255-1297        `weighted_gradient!` (boundary gradient
                                             zero: no open sides)
  src/operators/advection/cell_advection.jl:128-131, 205-220
                                             `enforce_no_permeation!`, `divergence!`
  src/navier_stokes/projection.jl:56-98      `_accumulate_pressure_increment!`
  src/navier_stokes/projection.jl:100-118    `_projection_compatibility!`
  src/navier_stokes/projection.jl:130-156    `_projection_rhs!`
  src/navier_stokes/projection.jl:221-260    `_project_prepared!`

Per-cell and per-face arithmetic follows the reference operation for operation
(no fused multiply-adds; divergence contributions summed per cell in face
order), so the elementwise results are bit-comparable.  The metric product
K @ v is a scipy sparse product: rounding-level agreement only.
"""
from __future__ import annotations

import numpy as np

from .krylov import solve as _solve
from .operator import remove_component_volume_means

EPS = np.finfo(np.float64).eps


def conditional_fraction(raw, floor=np.sqrt(EPS)):
    """`_refresh_conditional_fraction!` without embedded geometry: the
    physical fraction clamped to [0, 1] and the conditional fraction with the
    floor applied (<= floor -> 0, >= 1 - floor -> 1).  Raises ValueError like
    the reference's bounds check (finite, within 128 eps of [0, 1])."""
    raw = np.asarray(raw, dtype=np.float64)
    if not (np.isfinite(floor) and 0 < floor < 0.5):
        raise ValueError("fraction_floor must be finite and in (0, 0.5)")
    tol = 128 * EPS
    bad = ~np.isfinite(raw) | (raw < -tol) | (raw > 1 + tol)
    if np.any(bad):
        raise ValueError("volume fraction out of [0, 1]")
    value = np.clip(raw, 0.0, 1.0)
    ratio = value.copy()
    low = ratio <= floor
    high = ~low & (ratio >= 1 - floor)
    value[low] = 0.0
    ratio[low] = 0.0
    value[high] = 1.0
    ratio[high] = 1.0
    return value, ratio


def face_coefficients(mesh, conditional, density):
    """kappa_f = 1 / (rho_l c_f + rho_g (1 - c_f)), c_f the spacing-weighted
    mean of the two conditional fractions clamped to [0, 1]."""
    if not all(np.isfinite(r) and r > 0 for r in density):
        raise ValueError("phase densities must be finite and positive")
    nx, ny = mesh.block_size
    bm = mesh.face_minus // (nx * ny)
    bp = mesh.face_plus // (nx * ny)
    a = mesh.face_axis.astype(np.int64) - 1
    hm = mesh.spacing[bm, a]
    hp = mesh.spacing[bp, a]
    c = np.clip((hm * conditional[mesh.face_minus] + hp * conditional[mesh.face_plus]) / (hm + hp), 0.0, 1.0)
    rho = density[0] * c + density[1] * (1 - c)
    return 1.0 / rho


def surface_tension_jumps(mesh, conditional, sigma, curvature, formulation="cgfm"):
    """`_surface_tension_jumps!` with a constant curvature: sigma * kappa *
    jump * |f|, jump = [c+ > 1/2] - [c- > 1/2] (CGFM) or c+ - c- (CSF); zero
    where sigma or the jump is zero."""
    if not (np.isfinite(sigma) and sigma >= 0):
        raise ValueError("sigma must be finite and nonnegative")
    if not np.isfinite(curvature):
        raise ValueError("constant curvature must be finite")
    cm = conditional[mesh.face_minus]
    cp = conditional[mesh.face_plus]
    if formulation == "cgfm":
        jump = (cp > 0.5).astype(np.float64) - (cm > 0.5).astype(np.float64)
    elif formulation == "csf":
        jump = cp - cm
    else:
        raise ValueError("formulation must be CSF() or CGFM()")
    out = sigma * curvature * jump * mesh.face_area
    out[(jump == 0) | (sigma == 0)] = 0.0
    return out


def weighted_jump_force(op, jumps):
    """`_weighted_jump_force!`: interior sqrt(k) K (sqrt(k) j); boundary 0."""
    interior = op.sqrt_kappa * (op.K @ (op.sqrt_kappa * jumps))
    return interior, np.zeros(len(op.mesh.bface_cell))


def weighted_gradient(op, p):
    """`weighted_gradient!`: interior sqrt(k) K sqrt(k) |f| (p+ - p-); on a
    boundary face `_elliptic_boundary_gradient!` (elliptic.jl:1254-1262),
    -side * (2 k_b / h) * p on open faces and -side * 0 * p on closed ones."""
    mesh = op.mesh
    interior = op.weighted_gradient(p)
    boundary = (-mesh.bface_side.astype(np.float64) * op.boundary_gradient) * p[mesh.bface_cell]
    return interior, boundary


def divergence(mesh, u_interior, u_boundary):
    """`divergence!`: per cell, in face order, + u|f|/V on the minus cell and
    (-u|f|)/V on the plus cell of every interior face, then side u |f| / V of
    every boundary face."""
    vol = mesh.cell_volumes()
    flux = u_interior * mesh.face_area
    nf = len(flux)
    cells = np.empty(2 * nf, dtype=np.int64)
    vals = np.empty(2 * nf)
    cells[0::2] = mesh.face_minus
    cells[1::2] = mesh.face_plus
    vals[0::2] = flux / vol[mesh.face_minus]
    vals[1::2] = -flux / vol[mesh.face_plus]
    out = np.zeros(mesh.ncells)
    np.add.at(out, cells, vals)  # unbuffered: sequential in the listed order
    bflux = mesh.bface_side.astype(np.float64) * u_boundary * mesh.bface_area
    np.add.at(out, mesh.bface_cell, bflux / vol[mesh.bface_cell])
    return out


def projection_rhs(div, dt, inherited=None, reference_dt=None):
    """`_projection_rhs!`: -div / dt, plus ((ref_dt - dt) / (dt ref_dt)) times
    the inherited divergence on a shortened step."""
    out = -div / dt
    if inherited is not None:
        weight = (reference_dt - dt) / (dt * reference_dt)
        out = out + weight * inherited
    return out


def accumulate_pressure(op, pressure, increment):
    """`_accumulate_pressure_increment!`: p += phi, then on split domains each
    ungauged component's volume mean of p is removed (cells of no component: 0)."""
    p = pressure + increment
    comp = op.components
    if op.singular and len(comp["anchors"]) > 1:
        p = remove_component_volume_means(p, op.volumes, comp)
    return p


class ProjectionStats:
    def __init__(self, stats, dt, tolerance):
        self.solve = stats
        self.residual_scale = 1.0 / dt ** 2
        stats.residual_scale = self.residual_scale
        # the largest removed component mean (a non-finite one wins)
        m = 0.0
        for v in stats.removed_rhs_component_means:
            v = abs(v)
            if not np.isfinite(v) or v > m:
                m = v
        self.scaled_rhs_mean = 0.0 if m == 0 else dt ** 2 * m
        self.compatible = self.scaled_rhs_mean <= tolerance
        self.converged = stats.converged
        self.cycles = stats.cycles


def project(op, mg, u_interior, u_boundary, pressure, dt, *, tolerance=np.sqrt(EPS), max_cycles=100,
            compatibility="project", inherited=None, reference_dt=None, prepared=False):
    """`project!` (velocity_boundary = nothing: no-permeation boundary) or, with
    prepared=True, `_project_prepared!`.  Returns (u_interior, u_boundary,
    pressure, increment, stats); the increment solves the compatible
    projection of -D G_k phi = -D u* / dt with rtol 0, atol tolerance / dt^2."""
    if compatibility not in ("project", "error"):
        raise ValueError("compatibility must be :project or :error")
    if not dt > 0:
        raise ValueError("dt must be strictly positive")
    reference_dt = dt if reference_dt is None else reference_dt
    if not (np.isfinite(reference_dt) and reference_dt >= dt):
        raise ValueError("reference dt must be finite and at least dt")
    if not (np.isfinite(tolerance) and 0 < tolerance < 1):
        raise ValueError("tolerance must be finite and lie in (0, 1)")
    u_int = np.array(u_interior, dtype=np.float64)
    nb = len(op.mesh.bface_cell)
    u_bnd = np.zeros(nb) if u_boundary is None or np.ndim(u_boundary) == 0 \
        else np.array(u_boundary, dtype=np.float64)
    if not prepared:
        # no permeation through the closed sides; open faces keep their
        # velocity (`enforce_velocity_boundary!(...; preserve_open = true)`)
        from .operator import open_face_mask
        u_bnd[~open_face_mask(op.mesh, op.open_sides)] = 0.0
    b = projection_rhs(divergence(op.mesh, u_int, u_bnd), dt, inherited, reference_dt)
    phi, st = _solve(op, mg, b, np.zeros(op.mesh.ncells), rtol=0.0, atol=tolerance / dt ** 2,
                     max_cycles=max_cycles, compatibility=compatibility)
    g_int, g_bnd = weighted_gradient(op, phi)
    u_int = u_int - dt * g_int
    u_bnd = u_bnd - dt * g_bnd
    p = accumulate_pressure(op, np.asarray(pressure, dtype=np.float64), phi)
    return u_int, u_bnd, p, phi, ProjectionStats(st, dt, tolerance)
