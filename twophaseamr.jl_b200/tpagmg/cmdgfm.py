"""The linear solve of the CMDGFM two-velocity projection on the GPU.

TwoPhaseAMR.jl's `CMDGFMProjectionSolver` assembles a nonsymmetric two-block
system [A B; C J] [p; xi] = [f; g] -- pressure increments of the retained
cells of the gauge partition, then one jump per mixed face
(src/two_phase/projection/cmdgfm_projection.jl:1484-1592) -- and solves it in
`_project_cmdgfm_assembled!` (:2201-2291) with residual replacement around
BiCGSTAB, preconditioned by one V-cycle of the pressure hierarchy on the
reduced pressure block and an incomplete LU of J - C D^-1 B on the jump block.
`solve_cmdgfm` runs that solve on the device: the caller assembles the system
(as the reference does) and passes it with the `EllipticSolver` whose operator
is the system's pressure operator; its hierarchy is the pressure block's
preconditioner.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib


@dataclass
class CMDGFMSystem:
    """The assembled system as plain arrays (`tpa_cmdgfm_system`).

    row_ptr, col, val: the n x n matrix in CSR (columns increasing within a
    row), rows and columns the np pressure unknowns then the nx jumps.
    pressure_cell / pressure_anchor: the cell of every pressure unknown and the
    anchor cell of its component.  defect_weight: per row, dt^2 / V (pressure)
    or dt^2 / h (jump).  extra_*: the omitted anchor rows over the same
    unknowns.  row_scale, col_scale: the diagonal scalings D_r, D_c."""
    np_: int
    row_ptr: np.ndarray
    col: np.ndarray
    val: np.ndarray
    rhs: np.ndarray
    pressure_cell: np.ndarray
    pressure_anchor: np.ndarray
    defect_weight: np.ndarray
    extra_row_ptr: np.ndarray
    extra_col: np.ndarray
    extra_val: np.ndarray
    extra_rhs: np.ndarray
    extra_weight: np.ndarray
    row_scale: np.ndarray
    col_scale: np.ndarray
    drop_tolerance: float = 1e-3
    tolerance: float = float(np.sqrt(np.finfo(np.float64).eps))
    max_iterations: int = 500
    warm_start: bool = False          # `_cmdgfm_initial_solution!` (the reference's default is on)
    initial_pressure: np.ndarray = None  # np: the previous increment, reduced (x[cell] - x[anchor])

    @property
    def n(self):
        return len(self.row_ptr) - 1

    @property
    def nx(self):
        return self.n - self.np_

    def _c(self, precision):
        """The C struct and the arrays it points into (kept alive together)."""
        keep = dict(
            row_ptr=np.ascontiguousarray(self.row_ptr, dtype=np.int64),
            col=np.ascontiguousarray(self.col, dtype=np.int32),
            val=_lib.f64(self.val), rhs=_lib.f64(self.rhs),
            pressure_cell=np.ascontiguousarray(self.pressure_cell, dtype=np.int32),
            pressure_anchor=np.ascontiguousarray(self.pressure_anchor, dtype=np.int32),
            defect_weight=_lib.f64(self.defect_weight),
            extra_row_ptr=np.ascontiguousarray(self.extra_row_ptr, dtype=np.int64),
            extra_col=np.ascontiguousarray(self.extra_col, dtype=np.int32),
            extra_val=_lib.f64(self.extra_val), extra_rhs=_lib.f64(self.extra_rhs),
            extra_weight=_lib.f64(self.extra_weight),
            row_scale=_lib.f64(self.row_scale), col_scale=_lib.f64(self.col_scale),
            initial_pressure=(_lib.f64(self.initial_pressure) if self.initial_pressure is not None
                              else np.zeros(0)))
        c = _lib.CmdgfmSystemC()
        c.np, c.nx, c.na = int(self.np_), int(self.nx), int(len(keep["extra_row_ptr"]) - 1)
        for name, arr in keep.items():
            setattr(c, name, arr.ctypes.data if arr.size else None)
        c.drop_tolerance, c.tolerance = float(self.drop_tolerance), float(self.tolerance)
        c.max_iterations, c.precision = int(self.max_iterations), int(precision)
        c.warm_start = 1 if self.warm_start else 0
        return c, keep


@dataclass
class CMDGFMStats:
    """The linear part of `CMDGFMProjectionStats` (cmdgfm_projection.jl:315-340)."""
    converged: bool
    iterations: int
    attempts: int
    initial_residual: float
    final_residual: float
    pressure_defect: float
    jump_defect: float
    anchor_defect: float
    setup_ms: float
    device_ms: float
    kernel_launches: int
    factor_entries: int
    lower_levels: int
    upper_levels: int
    inverse_entries: int
    initial_guess_used: bool


_PRECISION = {"fp64": 0, "mixed": 1}


def solve_cmdgfm(solver, system: CMDGFMSystem, precision="fp64"):
    """Solve the assembled CMDGFM system on the GPU: returns (solution, stats).
    `precision` selects the V-cycle of the pressure block (the Krylov vectors
    are FP64 either way)."""
    if precision not in _PRECISION:
        raise ValueError("precision must be 'fp64' or 'mixed'")
    c, keep = system._c(_PRECISION[precision])
    x = np.zeros(system.n)
    st = _lib.CmdgfmStatsC()
    solver.ctx.call("tpa_cmdgfm_solve", C.byref(c), _lib.ptr(x, C.c_double), C.byref(st))
    del keep
    return x, CMDGFMStats(bool(st.converged), st.iterations, st.attempts, st.initial_residual, st.final_residual,
                          st.pressure_defect, st.jump_defect, st.anchor_defect, st.setup_ms, st.device_ms,
                          st.kernel_launches, st.factor_entries, st.lower_levels, st.upper_levels,
                          st.inverse_entries, bool(st.initial_guess_used))


def cmdgfm_factor(system: CMDGFMSystem):
    """The host set-up alone (no GPU): the Schur complement S = J - C D^-1 B
    and its incomplete LU factors L (strictly lower) and U (pivot first in each
    row), each as (row_ptr, col, val)."""
    c, keep = system._c(0)
    lib = _lib.lib()
    counts = [C.c_int64() for _ in range(3)]
    code = lib.tpa_cmdgfm_factor(C.byref(c), C.byref(counts[0]), None, None, None, C.byref(counts[1]), None, None,
                                 None, C.byref(counts[2]), None, None, None)
    if code:
        raise _lib.TpaError(code, "tpa_cmdgfm_factor failed")
    nx = system.nx
    out = [(np.empty(nx + 1, dtype=np.int64), np.empty(k.value, dtype=np.int32), np.empty(k.value))
           for k in counts]
    args = []
    for cnt, (ptr, col, val) in zip(counts, out):
        args += [C.byref(cnt), _lib.ptr(ptr, C.c_int64), _lib.ptr(col, C.c_int32), _lib.ptr(val, C.c_double)]
    code = lib.tpa_cmdgfm_factor(C.byref(c), *args)
    if code:
        raise _lib.TpaError(code, "tpa_cmdgfm_factor failed")
    del keep
    return out
