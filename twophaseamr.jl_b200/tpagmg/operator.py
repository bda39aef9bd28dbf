"""`PoissonOperator` and the two-phase coefficient / surface-tension inputs.

Mirrors (ronaldremmerswaal/TwoPhaseAMR.jl):
  src/operators/elliptic.jl:969-980     PoissonOperator(mesh; face_coefficient, velocity_boundary,
                                        boundary_face_coefficient)
  src/operators/elliptic.jl:76-87       `_pressure_boundary_sides` (open sides)
  src/two_phase/forces.jl:23-36, 69-84  staggered liquid fraction, mixture density
  src/two_phase/forces.jl:113-140       PoissonOperator(interface; density): kappa = 1/rho_f
  src/two_phase/forces.jl:312-314, 345-378  CGFM jumps sigma*kappa*([c+ > 1/2] - [c- > 1/2])*|f|

The operator's matrix lives in the B200 library; this object holds the face
coefficients and validates them as the reference constructor does.
"""
from __future__ import annotations

import numpy as np


OPEN_CONDITIONS = ("outflow", "zero_gradient")
SIDES = ("left", "right", "bottom", "top")


def pressure_boundary_sides(velocity_boundary):
    """`_pressure_boundary_sides` (elliptic.jl:76-87): which sides (left, right,
    bottom, top) are open.  None, "no_slip" or "free_slip": none.  A 4-tuple of
    booleans is taken as it is; a dict maps side names to velocity conditions
    ("outflow" and "zero_gradient" open a side, any other closes it)."""
    if velocity_boundary is None or velocity_boundary in ("no_slip", "free_slip"):
        return (False, False, False, False)
    if isinstance(velocity_boundary, dict):
        unknown = set(velocity_boundary) - set(SIDES)
        if unknown:
            raise ValueError(f"unknown sides: {sorted(unknown)}")
        return tuple(velocity_boundary.get(side) in OPEN_CONDITIONS for side in SIDES)
    sides = tuple(bool(v) for v in velocity_boundary)
    if len(sides) != 4:
        raise ValueError("velocity_boundary needs four sides (left, right, bottom, top)")
    return sides


class PoissonOperator:
    """Positive Poisson operator `-div(kappa grad p)` on a `BlockTreeMesh`.

    velocity_boundary: the open (pressure Dirichlet) sides, see
    `pressure_boundary_sides`; boundary_face_coefficient: one per boundary face
    for the open faces, or None to extend the interior coefficients."""

    def __init__(self, mesh, face_coefficient=1.0, velocity_boundary=None, boundary_face_coefficient=None):
        self.mesh = mesh
        self.open_sides = pressure_boundary_sides(velocity_boundary)
        for a in (0, 1):
            if mesh.periodic[a] and (self.open_sides[2 * a] or self.open_sides[2 * a + 1]):
                raise ValueError("a periodic axis has no open sides")
        self.boundary_face_coefficient = None
        if boundary_face_coefficient is not None:
            nb = mesh.nboundary_faces
            bc = np.full(nb, float(boundary_face_coefficient)) if np.isscalar(boundary_face_coefficient) \
                else np.array(boundary_face_coefficient, dtype=np.float64)
            if bc.shape != (nb,):
                raise ValueError("one coefficient and aperture are required per boundary face")
            if not (np.all(np.isfinite(bc)) and np.all(bc >= 0)):
                raise ValueError("boundary coefficients must be finite and nonnegative")
            self.boundary_face_coefficient = bc
        nf = mesh.nfaces
        if np.isscalar(face_coefficient):
            kappa = np.full(nf, float(face_coefficient))
        elif callable(face_coefficient):
            cx, cy = mesh.face_centers()
            kappa = np.array([float(face_coefficient(x, y, a)) for x, y, a in zip(cx, cy, mesh.face_axis)])
        else:
            kappa = np.array(face_coefficient, dtype=np.float64)
            if kappa.shape != (nf,):
                raise ValueError("one coefficient is required per interior face")
        if not np.all(np.isfinite(kappa)):
            raise ValueError("face coefficients must be finite")
        if np.any(kappa < 0):
            raise ValueError("face coefficients must be nonnegative")
        self.face_coefficient = kappa
        self.volumes = mesh.cell_volumes()
        self.reaction = 0.0
        self.diffusion = 1.0

    @classmethod
    def two_phase(cls, mesh, fraction, density=(1.0, 1.0)):
        """`PoissonOperator(interface; density)` from cell liquid fractions."""
        return cls(mesh, 1.0 / mixture_density(mesh, fraction, density))


def staggered_liquid_fraction(mesh, fraction):
    """`_staggered_liquid_fraction` (forces.jl:23-36): spacing-weighted mean of
    the two cell fractions, clamped to [0, 1]."""
    nx, ny = mesh.block_size
    bm = mesh.face_minus // (nx * ny)
    bp = mesh.face_plus // (nx * ny)
    a = mesh.face_axis.astype(np.int64) - 1
    hm = mesh.spacing[bm, a]
    hp = mesh.spacing[bp, a]
    c = (hm * fraction[mesh.face_minus] + hp * fraction[mesh.face_plus]) / (hm + hp)
    return np.clip(c, 0.0, 1.0)


def mixture_density(mesh, fraction, density):
    """`_mixture_density!` (forces.jl:69-84): rho_l c + rho_g (1 - c) per face."""
    if not all(np.isfinite(r) and r > 0 for r in density):
        raise ValueError("phase densities must be finite and positive")
    c = staggered_liquid_fraction(mesh, np.asarray(fraction, dtype=np.float64))
    return density[0] * c + density[1] * (1 - c)


def surface_tension_jumps(mesh, fraction, sigma, curvature):
    """`_surface_tension_jumps!` with the CGFM jump and a constant curvature
    (forces.jl:312-314, 345-378): sigma * kappa * ([c+ > 1/2] - [c- > 1/2]) * |f|."""
    if not (np.isfinite(sigma) and sigma >= 0):
        raise ValueError("sigma must be finite and nonnegative")
    if not np.isfinite(curvature):
        raise ValueError("constant curvature must be finite")
    f = np.asarray(fraction, dtype=np.float64)
    jump = (f[mesh.face_plus] > 0.5).astype(np.float64) - (f[mesh.face_minus] > 0.5).astype(np.float64)
    out = sigma * curvature * jump * mesh.face_area
    out[(jump == 0) | (sigma == 0)] = 0.0
    return out
