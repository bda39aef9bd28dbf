"""The one-velocity projection step around the pressure solve, on the B200.

Mirrors (ronaldremmerswaal/TwoPhaseAMR.jl):
  src/navier_stokes/projection.jl:183-260       project!(velocity, pressure, solver, dt, workspace;
        tolerance=sqrt(eps), max_cycles=100, compatibility=:project) and `_project_prepared!`
  src/operators/advection/cell_advection.jl:205-220  divergence!(destination, velocity)
  src/operators/elliptic.jl:1272-1297            weighted_gradient!(destination, pressure, operator, workspace)
  src/two_phase/forces.jl:328-342                surface_tension!(acceleration, interface, operator, workspace;
        sigma, formulation=CGFM(), curvature)  (constant curvature)
  src/two_phase/forces.jl:113-140                PoissonOperator(field; density): kappa = 1/rho_f
  src/interface/interface_field.jl:248-291       `_refresh_conditional_fraction!`

`FaceVelocity` holds host arrays (`interior` per interior face, `boundary`
per boundary face); the host-array functions copy to the device and back.
The `*_device` functions take torch CUDA tensors and keep everything resident,
so a two-phase step (fractions -> coefficients -> refresh -> force ->
projection) makes no host copies of its fields.  No CPU path exists: every
function runs the library's kernels.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _lib
from .solver import _PRECISION, _compat

FRACTION_FLOOR = float(np.sqrt(np.finfo(np.float64).eps))  # InterfaceField's default floor
DEFAULT_TOLERANCE = float(np.sqrt(np.finfo(np.float64).eps))  # project!'s default tolerance
_FORMULATION = {"cgfm": 0, "csf": 1}


class FaceVelocity:
    """`FaceVelocity(mesh)`: face-normal velocity on interior and boundary faces."""

    def __init__(self, mesh, interior=None, boundary=None):
        self.mesh = mesh
        self.interior = np.zeros(mesh.nfaces) if interior is None else _lib.f64(interior).copy()
        self.boundary = np.zeros(mesh.nboundary_faces) if boundary is None else _lib.f64(boundary).copy()
        if self.interior.shape != (mesh.nfaces,) or self.boundary.shape != (mesh.nboundary_faces,):
            raise ValueError("face velocity sizes do not match the mesh")


class ProjectionOptions(C.Structure):
    """`tpa_projection_options`."""

    _fields_ = [("dt", C.c_double), ("tolerance", C.c_double), ("reference_dt", C.c_double),
                ("inherited_divergence", C.c_void_p), ("max_cycles", C.c_int32), ("compatibility", C.c_int32),
                ("precision", C.c_int32), ("prepared", C.c_int32)]


def _options(solver, dt, tolerance, max_cycles, compatibility, precision, prepared, reference_dt, inherited_ptr):
    if reference_dt is not None and float(reference_dt) == 0.0:
        # 0 means "not given" at the C-ABI; an explicit 0 is below dt
        raise ValueError("reference dt must be finite and at least dt")
    return ProjectionOptions(float(dt), float(tolerance), 0.0 if reference_dt is None else float(reference_dt),
                             inherited_ptr,
                             int(max_cycles), _compat(compatibility), _PRECISION[precision or solver.precision],
                             1 if prepared else 0)


def _stats(solver, st):
    return dataclasses.replace(solver._stats_from(st))


def _torch():
    import torch
    return torch


def _dev(a, torch, device):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(device)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


# ---- host-array API --------------------------------------------------------------

def project(velocity, pressure, solver, dt, *, tolerance=DEFAULT_TOLERANCE, max_cycles=100, compatibility="project",
            precision=None, prepared=False, inherited_divergence=None, reference_dt=None):
    """`project!`: overwrites `velocity` (a FaceVelocity) and `pressure` (a
    cell array) in place and returns the increment solve's LinearSolverStats
    (residual_scale 1/dt^2; `compatible` from dt^2 times the removed mean).
    `prepared=True` is `_project_prepared!` (boundary velocity kept)."""
    if not isinstance(pressure, np.ndarray) or pressure.dtype != np.float64 or not pressure.flags.c_contiguous:
        raise TypeError("pressure must be a contiguous float64 array (updated in place)")
    inh = None if inherited_divergence is None else _lib.f64(inherited_divergence)
    opts = _options(solver, dt, tolerance, max_cycles, compatibility, precision, prepared, reference_dt,
                    inh.ctypes.data if inh is not None else None)
    st = _lib.StatsC()
    solver.ctx.call("tpa_project", _lib.ptr(velocity.interior, C.c_double), _lib.ptr(velocity.boundary, C.c_double),
                    _lib.ptr(pressure, C.c_double), C.byref(opts), C.byref(st))
    return _stats(solver, st)


def _host_call(solver, fn, inputs, outputs):
    torch = _torch()
    dev = f"cuda:{solver.device}"
    ins = [_dev(a, torch, dev) if a is not None else None for a in inputs]
    outs = [torch.empty(n, dtype=torch.float64, device=dev) for n in outputs]
    fn(*ins, *outs)
    return [o.cpu().numpy() for o in outs]


def divergence(velocity, solver):
    """`divergence!` of a FaceVelocity: cell array."""
    (d,) = _host_call(solver, lambda u, b, out: divergence_device(solver, u, b, out),
                      [velocity.interior, velocity.boundary], [solver.operator.mesh.ncells])
    return d


def weighted_gradient(pressure, solver):
    """`weighted_gradient!`: a FaceVelocity."""
    mesh = solver.operator.mesh
    g, gb = _host_call(solver, lambda p, gi, gbd: weighted_gradient_device(solver, p, gi, gbd),
                       [pressure], [mesh.nfaces, mesh.nboundary_faces])
    return FaceVelocity(mesh, g, gb)


def conditional_fraction(fraction, solver, fraction_floor=FRACTION_FLOOR):
    """(physical, conditional) fractions of `_refresh_conditional_fraction!`."""
    n = solver.operator.mesh.ncells
    return tuple(_host_call(solver, lambda f, ph, co: conditional_fraction_device(solver, f, co, ph, fraction_floor),
                            [fraction], [n, n]))


def face_coefficients(conditional, solver, density):
    """kappa_f = 1/rho_f of `PoissonOperator(field; density)`."""
    (k,) = _host_call(solver, lambda c, out: face_coefficients_device(solver, c, density, out), [conditional],
                      [solver.operator.mesh.nfaces])
    return k


def surface_tension(conditional, solver, *, sigma, curvature, formulation="cgfm"):
    """`surface_tension!` with a constant curvature: a FaceVelocity
    (acceleration) from the conditional fractions."""
    mesh = solver.operator.mesh
    a, ab = _host_call(solver, lambda c, ai, abd: surface_tension_device(solver, c, ai, abd, sigma=sigma,
                                                                          curvature=curvature,
                                                                          formulation=formulation),
                       [conditional], [mesh.nfaces, mesh.nboundary_faces])
    return FaceVelocity(mesh, a, ab)


# ---- device-array API (torch CUDA float64 tensors) ----------------------------------

def _sync_stream(solver):
    torch = _torch()
    solver.set_stream(torch.cuda.current_stream(solver.device).cuda_stream)


def conditional_fraction_device(solver, fraction, conditional, physical=None, fraction_floor=FRACTION_FLOOR):
    _sync_stream(solver)
    solver.ctx.call("tpa_conditional_fraction_device", _ptr(fraction), float(fraction_floor), _ptr(physical),
                    _ptr(conditional))


def face_coefficients_device(solver, conditional, density, kappa):
    _sync_stream(solver)
    solver.ctx.call("tpa_face_coefficients_device", _ptr(conditional), float(density[0]), float(density[1]),
                    _ptr(kappa))


def surface_tension_device(solver, conditional, accel_interior, accel_boundary=None, *, sigma, curvature,
                           formulation="cgfm"):
    if formulation not in _FORMULATION:
        raise ValueError("formulation must be CSF() or CGFM()")
    _sync_stream(solver)
    solver.ctx.call("tpa_surface_tension_device", _ptr(conditional), float(sigma), float(curvature),
                    _FORMULATION[formulation], _ptr(accel_interior), _ptr(accel_boundary))


def weighted_gradient_device(solver, pressure, grad_interior, grad_boundary=None):
    _sync_stream(solver)
    solver.ctx.call("tpa_weighted_gradient_device", _ptr(pressure), _ptr(grad_interior), _ptr(grad_boundary))


def divergence_device(solver, u_interior, u_boundary, out):
    _sync_stream(solver)
    solver.ctx.call("tpa_divergence_device", _ptr(u_interior), _ptr(u_boundary), _ptr(out))


def project_device(u_interior, u_boundary, pressure, solver, dt, *, tolerance=DEFAULT_TOLERANCE, max_cycles=100,
                   compatibility="project", precision=None, prepared=False, inherited_divergence=None,
                   reference_dt=None):
    """`project!` on device tensors (updated in place)."""
    _sync_stream(solver)
    opts = _options(solver, dt, tolerance, max_cycles, compatibility, precision, prepared, reference_dt,
                    inherited_divergence.data_ptr() if inherited_divergence is not None else None)
    st = _lib.StatsC()
    solver.ctx.call("tpa_project_device", _ptr(u_interior), _ptr(u_boundary), _ptr(pressure), C.byref(opts),
                    C.byref(st))
    return _stats(solver, st)


def refresh_device(solver, kappa):
    """`_refresh_geometric_multigrid!` from device face coefficients."""
    _sync_stream(solver)
    solver.ctx.call("tpa_refresh_device", _ptr(kappa))
    solver.operator.face_coefficient = kappa.detach().cpu().numpy()


class TwoPhaseStep:
    """The device-resident pressure part of a one-velocity two-phase step:
    liquid fractions -> conditional fractions -> kappa = 1/rho_f -> hierarchy
    refresh -> CGFM / CSF force -> projection, all on the GPU
    (two_phase/stepping.jl:73-111 calls these in this order)."""

    def __init__(self, solver, density, *, sigma, curvature, formulation="cgfm", fraction_floor=FRACTION_FLOOR):
        torch = _torch()
        mesh = solver.operator.mesh
        dev = f"cuda:{solver.device}"
        self.solver, self.density = solver, tuple(density)
        self.sigma, self.curvature, self.formulation, self.floor = sigma, curvature, formulation, fraction_floor
        f64 = dict(dtype=torch.float64, device=dev)
        self.conditional = torch.zeros(mesh.ncells, **f64)
        self.physical = torch.zeros(mesh.ncells, **f64)
        self.kappa = torch.zeros(mesh.nfaces, **f64)
        self.accel = torch.zeros(mesh.nfaces, **f64)
        self.accel_boundary = torch.zeros(max(mesh.nboundary_faces, 1), **f64)

    def update_interface(self, fraction):
        """New liquid fractions (device tensor): coefficients and the
        multigrid hierarchy follow."""
        s = self.solver
        conditional_fraction_device(s, fraction, self.conditional, self.physical, self.floor)
        face_coefficients_device(s, self.conditional, self.density, self.kappa)
        refresh_device(s, self.kappa)

    def force(self):
        surface_tension_device(self.solver, self.conditional, self.accel, self.accel_boundary, sigma=self.sigma,
                               curvature=self.curvature, formulation=self.formulation)
        return self.accel

    def project(self, u_interior, u_boundary, pressure, dt, **kw):
        return project_device(u_interior, u_boundary, pressure, self.solver, dt, **kw)
