"""`EllipticSolver` and `solve` (the reference's `solve!`) on the B200.

Mirrors (ronaldremmerswaal/TwoPhaseAMR.jl):
  src/solvers/multigrid/elliptic_solver.jl:211-302  EllipticSolver(operator; krylov,
        preconditioner, preconditioner_options, multigrid)
  src/solvers/multigrid/elliptic_solver.jl:614-675  solve!(solution, solver, rhs;
        rtol=1e-10, atol=0, max_cycles=100, compatibility=:project)
  src/solvers/multigrid/stats.jl:100-135            LinearSolverStats
  src/solvers/multigrid/cycles.jl:328-340           CG needs equal pre/post sweeps

The hierarchy is built on the host by the library; every solve runs on the GPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .options import LinearSolverOptions, MultigridOptions

# "fp64": FP64 V-cycle and Krylov vectors; "mixed": FP32 V-cycle, FP64 Krylov
# vectors; "mixed_ir": FP32 V-cycle and Krylov vectors (r, p, Ap, z) in an FP64
# iterative-refinement loop (FP64 iterate, true residual and inner products)
_PRECISION = {"fp64": 0, "mixed": 1, "mixed_ir": 2}


@dataclass
class LinearSolverStats:
    """Convergence statistics of the latest solve (stats.jl:113-135)."""

    cycles: int = 0
    converged: bool = False
    compatible: bool = True
    initial_l2: float = float("inf")
    initial_linf: float = float("inf")
    final_l2: float = float("inf")
    final_linf: float = float("inf")
    target_linf: float = float("inf")
    residual_scale: float = 1.0
    removed_rhs_mean: float = 0.0
    removed_rhs_component_means: list = field(default_factory=list)
    removed_rhs_component_anchors: list = field(default_factory=list)
    method: str = "cg"
    preconditioner: str = "gpu_tree_geometric_multigrid"
    device_ms: float = 0.0
    restarts: int = 0
    kernel_launches: int = 0
    precision: str = "fp64"


class EllipticSolver:
    """Krylov CG + tree geometric multigrid on one B200 for a `PoissonOperator`."""

    def __init__(self, operator, *, krylov=None, krylov_options=None, preconditioner="gpu_tree_geometric",
                 preconditioner_options=None, multigrid=None, coarse_size=None, pre_sweeps=None,
                 post_sweeps=None, max_levels=None, device=0, options=None):
        if options is not None:
            if not isinstance(options, LinearSolverOptions):
                raise TypeError("options must be LinearSolverOptions")
            krylov, krylov_options = options.krylov, options.krylov_options
            preconditioner, preconditioner_options = options.preconditioner, options.preconditioner_options
        if preconditioner == "auto":
            preconditioner = "gpu_tree_geometric"
        if preconditioner not in ("geometric", "tree_geometric", "gpu_tree_geometric"):
            raise ValueError("the B200 solver implements the tree geometric multigrid preconditioner only")
        if krylov not in (None, "cg", "CG"):
            raise ValueError("the B200 solver implements CG only")
        mg = multigrid or MultigridOptions()
        mg = MultigridOptions(coarse_size=mg.coarse_size if coarse_size is None else coarse_size,
                              pre_sweeps=mg.pre_sweeps if pre_sweeps is None else pre_sweeps,
                              post_sweeps=mg.post_sweeps if post_sweeps is None else post_sweeps,
                              max_levels=mg.max_levels if max_levels is None else max_levels,
                              smoother=mg.smoother)
        if mg.pre_sweeps != mg.post_sweeps:
            raise ValueError(f"CG requires equal pre_sweeps and post_sweeps for a geometric multigrid "
                             f"preconditioner; got {mg.pre_sweeps} and {mg.post_sweeps}")
        popts = dict(preconditioner_options or {})
        precision = popts.pop("precision", "fp64")
        if precision not in _PRECISION:
            raise ValueError("precision must be 'fp64', 'mixed' or 'mixed_ir'")
        if popts:
            raise ValueError(f"unsupported preconditioner_options: {sorted(popts)}")
        self.operator = operator
        self.multigrid = mg
        self.precision = precision
        mesh = operator.mesh
        self.device = int(device)
        self.ctx = _lib.Context(device)
        self.ctx.call("tpa_set_mesh", *mesh._mesh_args())
        self._kappa = _lib.f64(operator.face_coefficient)
        sides = getattr(operator, "open_sides", (False, False, False, False))
        if any(sides):
            so = np.array([1 if v else 0 for v in sides], dtype=np.int32)
            bc = getattr(operator, "boundary_face_coefficient", None)
            self._bcoef = None if bc is None else _lib.f64(bc)
            self.ctx.call("tpa_set_open_boundaries", _lib.ptr(so, C.c_int32),
                          None if self._bcoef is None else _lib.ptr(self._bcoef, C.c_double))
        self.ctx.call("tpa_set_operator", _lib.ptr(self._kappa, C.c_double))
        o = _lib.MultigridOptionsC(mg.coarse_size, mg.pre_sweeps, mg.post_sweeps, mg.max_levels,
                                   1 if mg.smoother == "red_black" else 0)
        self.ctx.call("tpa_build_hierarchy", C.byref(o))
        self.stats = LinearSolverStats(precision=precision)

    # -- hierarchy queries (parity tests) -------------------------------------
    def level_sizes(self):
        n = C.c_int32()
        self.ctx.call("tpa_hierarchy_sizes", C.byref(n), None, 0)
        sizes = np.zeros(n.value, dtype=np.int64)
        self.ctx.call("tpa_hierarchy_sizes", C.byref(n), _lib.ptr(sizes, C.c_int64), n.value)
        return [int(s) for s in sizes]

    def level_owners(self, level):
        out = np.zeros(self.level_sizes()[level], dtype=np.int32)
        self.ctx.call("tpa_level_owners", int(level), _lib.ptr(out, C.c_int32))
        return out

    def level_matrix(self, level=0):
        """The assembled operator of a level as (row_ptr, col, val) CSR arrays
        (int64, int32, float64) with sorted columns."""
        nnz = C.c_int64()
        self.ctx.call("tpa_level_matrix", int(level), C.byref(nnz), None, None, None)
        n = self.level_sizes()[level]
        row_ptr = np.empty(n + 1, dtype=np.int64)
        col = np.empty(nnz.value, dtype=np.int32)
        val = np.empty(nnz.value, dtype=np.float64)
        self.ctx.call("tpa_level_matrix", int(level), C.byref(nnz), _lib.ptr(row_ptr, C.c_int64),
                      _lib.ptr(col, C.c_int32), _lib.ptr(val, C.c_double))
        return row_ptr, col, val

    def level_info(self, level):
        sw, tw, nc = C.c_double(), C.c_double(), C.c_int32()
        self.ctx.call("tpa_level_info", int(level), C.byref(sw), C.byref(tw), C.byref(nc))
        return sw.value, tw.value, nc.value

    def level_red_black(self, level, ncells):
        """Red-black colours (0 red, 1 black) of a level and its half-sweep weight."""
        col = np.zeros(ncells, dtype=np.uint8)
        w = C.c_double()
        self.ctx.call("tpa_level_red_black", int(level), col.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(w))
        return col, w.value

    def level_face_coefficients(self, level, nfaces):
        out = np.zeros(nfaces, dtype=np.float64)
        self.ctx.call("tpa_level_face_coefficients", int(level), _lib.ptr(out, C.c_double))
        return out

    def device_info(self):
        """Device layout: structured levels, exception rows, tail start, fused cycle."""
        out = np.zeros(4, dtype=np.int64)
        self.ctx.call("tpa_device_info", _lib.ptr(out, C.c_int64))
        return {"structured_levels": int(out[0]), "exception_rows": int(out[1]),
                "tail_first_level": int(out[2]), "fused_cycle": bool(out[3])}

    # -- device layout ---------------------------------------------------------
    @staticmethod
    def _tune_dict(t):
        return {"tail_cells": t.tail_cells, "tail_ctas": t.tail_ctas, "structured": t.structured,
                "vectorized": t.vectorized, "pdl": t.pdl, "fuse_restrict": t.fuse_restrict, "persistent": t.persistent,
                "tiles": t.tiles, "ms_per_vcycle": t.ms_per_vcycle}

    def autotune(self, precision=None, vcycles=20):
        """Time the candidate device layouts of the V-cycle and keep the
        fastest; returns (best, every measurement) as dicts."""
        best = _lib.TuneC()
        tried = (_lib.TuneC * 64)()
        n = C.c_int32()
        self.ctx.call("tpa_autotune", _PRECISION[precision or self.precision], int(vcycles), C.byref(best), tried,
                      64, C.byref(n))
        return self._tune_dict(best), [self._tune_dict(tried[k]) for k in range(n.value)]

    def tuning(self):
        t = _lib.TuneC()
        self.ctx.call("tpa_get_tuning", C.byref(t))
        return self._tune_dict(t)

    def tiled_levels(self):
        """Levels whose V-cycle phases run on haloed block tiles."""
        n = C.c_int32()
        self.ctx.call("tpa_tiled_levels", C.byref(n))
        return int(n.value)

    def streamed_levels(self):
        """Of the tiled levels, those on the row-streaming kernels (tiles 4, 5)."""
        n = C.c_int32()
        self.ctx.call("tpa_streamed_levels", C.byref(n))
        return int(n.value)

    def set_tuning(self, **fields):
        """Apply a layout (tail_cells, tail_ctas, structured, vectorized, pdl,
        fuse_restrict, persistent, tiles; omitted fields: default)."""
        keys = ("tail_cells", "tail_ctas", "structured", "vectorized", "pdl", "fuse_restrict", "persistent", "tiles")
        unknown = set(fields) - set(keys)
        if unknown:
            raise ValueError(f"unknown layout fields: {sorted(unknown)}")
        t = _lib.TuneC(*(int(fields.get(k, -1)) for k in keys), 0.0)
        self.ctx.call("tpa_set_tuning", C.byref(t))

    def residual_norms_device(self, r_ptr):
        """`_integrated_residual_norms` of an integrated residual held on the
        device (raw CUDA pointer, cell order): (L2, strong L-infinity)."""
        out = np.zeros(2)
        self.ctx.call("tpa_residual_norms", C.c_void_p(r_ptr), _lib.ptr(out, C.c_double))
        return float(out[0]), float(out[1])

    # -- device operations --------------------------------------------------
    def refresh(self, face_coefficient):
        """`_refresh_geometric_multigrid!` after a coefficient change."""
        self._kappa = _lib.f64(face_coefficient)
        self.ctx.call("tpa_refresh", _lib.ptr(self._kappa, C.c_double))
        self.operator.face_coefficient = self._kappa.copy()

    def last_refresh(self):
        """How the last `refresh` ran: ("host" | "device" | None, wall ms)."""
        path = C.c_int32()
        ms = C.c_double()
        self.ctx.call("tpa_last_refresh", C.byref(path), C.byref(ms))
        return {0: None, 1: "host", 2: "device"}[path.value], ms.value

    def apply(self, x):
        x = _lib.f64(x)
        y = np.empty_like(x)
        self.ctx.call("tpa_apply", _lib.ptr(x, C.c_double), _lib.ptr(y, C.c_double))
        return y

    def vcycle(self, r, precision=None):
        r = _lib.f64(r)
        z = np.empty_like(r)
        # the refinement solve preconditions with the FP32 cycle
        self.ctx.call("tpa_vcycle", _lib.ptr(r, C.c_double), _lib.ptr(z, C.c_double),
                      min(_PRECISION[precision or self.precision], 1))
        return z

    def _stats_from(self, st):
        s = self.stats
        s.cycles, s.converged, s.compatible = st.cycles, bool(st.converged), bool(st.compatible)
        s.initial_l2, s.initial_linf = st.initial_l2, st.initial_linf
        s.final_l2, s.final_linf, s.target_linf = st.final_l2, st.final_linf, st.target_linf
        s.residual_scale, s.removed_rhs_mean = st.residual_scale, st.removed_rhs_mean
        s.device_ms, s.restarts, s.kernel_launches = st.device_ms, st.restarts, st.kernel_launches
        return s

    # -- adjoint --------------------------------------------------------------
    def adjoint(self, p, pbar, *, rtol=1e-10, atol=0.0, max_cycles=100, precision=None):
        """Reverse-mode derivative of `solve!` at the solution p for the
        cotangent pbar = dJ/dp: returns (dJ/d strong rhs, dJ/d face
        coefficient, stats of the adjoint solve)."""
        p, pbar = _lib.f64(p), _lib.f64(pbar)
        n, nf = self.operator.mesh.ncells, self.operator.mesh.nfaces
        if p.shape != (n,) or pbar.shape != (n,):
            raise ValueError("solution and cotangent must be cell fields of the solver's mesh")
        rhs_bar = np.empty(n)
        kappa_bar = np.empty(nf)
        st = _lib.StatsC()
        self.ctx.call("tpa_adjoint", _lib.ptr(p, C.c_double), _lib.ptr(pbar, C.c_double),
                      _lib.ptr(rhs_bar, C.c_double), _lib.ptr(kappa_bar, C.c_double), float(rtol), float(atol),
                      int(max_cycles), _PRECISION[precision or self.precision], C.byref(st))
        return rhs_bar, kappa_bar, self._stats_from(st)

    def adjoint_device(self, p_ptr, pbar_ptr, rhs_bar_ptr, kappa_bar_ptr, *, rtol=1e-10, atol=0.0, max_cycles=100,
                       precision=None):
        """`adjoint` on device arrays (raw CUDA pointers; either output may be 0)."""
        st = _lib.StatsC()
        self.ctx.call("tpa_adjoint_device", C.c_void_p(p_ptr), C.c_void_p(pbar_ptr),
                      C.c_void_p(rhs_bar_ptr or None), C.c_void_p(kappa_bar_ptr or None), float(rtol), float(atol),
                      int(max_cycles), _PRECISION[precision or self.precision], C.byref(st))
        return self._stats_from(st)

    def face_coefficient_gradient(self, p, lam):
        """-lam' (dS/dkappa_f) p per interior face (the adjoint's face kernel)."""
        p, lam = _lib.f64(p), _lib.f64(lam)
        g = np.empty(self.operator.mesh.nfaces)
        self.ctx.call("tpa_face_coefficient_gradient", _lib.ptr(p, C.c_double), _lib.ptr(lam, C.c_double),
                      _lib.ptr(g, C.c_double))
        return g

    def set_stream(self, stream):
        """Order device work after the given CUDA stream handle (int; 0 = own)."""
        self.ctx.call("tpa_set_stream", C.c_void_p(int(stream) or None))

    def solve_device(self, rhs_ptr, x_ptr, *, rtol=1e-10, atol=0.0, max_cycles=100, compatibility="project",
                     precision=None):
        """`solve!` on device arrays (raw CUDA pointers, cell order)."""
        st = _lib.StatsC()
        self.ctx.call("tpa_solve_device", C.c_void_p(rhs_ptr), C.c_void_p(x_ptr), float(rtol), float(atol),
                      int(max_cycles), _compat(compatibility), _PRECISION[precision or self.precision], C.byref(st))
        return self._stats_from(st)


def _compat(compatibility):
    if compatibility not in ("project", "error"):
        raise ValueError("compatibility must be :project or :error")
    return 0 if compatibility == "project" else 1


class BatchResult(list):
    """Per-problem `LinearSolverStats` of a batched solve, plus `device_ms`:
    the device time from the batch's start to its last problem's end."""

    device_ms = 0.0


def solve_batched(solutions, solvers, rhs, *, rtol=1e-10, atol=0.0, max_cycles=100, compatibility="project",
                  precision="mixed", workers=32):
    """`solve!` for many independent problems at once (one `EllipticSolver`
    per problem; solvers must be distinct).  `solutions[k]` (initial guess in,
    solution out) and `rhs[k]` are float64 cell arrays of problem k: numpy
    arrays, or raw CUDA pointers (ints) on the solvers' device.  Returns a
    `BatchResult`; raises on the first failed problem after all have run."""
    count = len(solvers)
    if len(solutions) != count or len(rhs) != count:
        raise ValueError("one solution and one right-hand side are required per solver")
    if len({id(s) for s in solvers}) != count:
        raise ValueError("every problem needs its own solver")
    comp = _compat(compatibility)
    device = count > 0 and isinstance(solutions[0], int)
    if device:
        if not all(isinstance(v, int) for v in list(solutions) + list(rhs)):
            raise TypeError("device batches take raw pointers for every problem")
        rp = (C.c_void_p * count)(*rhs)
        xp = (C.c_void_p * count)(*solutions)
        entry = "tpa_solve_batched_device"
    else:
        bs = [_lib.f64(b) for b in rhs]
        for k, (x, s, b) in enumerate(zip(solutions, solvers, bs)):
            if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous):
                raise TypeError("solutions must be contiguous float64 arrays")
            n = s.operator.mesh.ncells
            if x.shape != (n,) or b.shape != (n,):
                raise ValueError(f"problem {k}: fields and multigrid solver must share a mesh")
        rp = (_lib.f64p * count)(*[_lib.ptr(b, C.c_double) for b in bs])
        xp = (_lib.f64p * count)(*[_lib.ptr(x, C.c_double) for x in solutions])
        entry = "tpa_solve_batched"
    ctxs = (C.c_void_p * count)(*[s.ctx.handle.value for s in solvers])
    stats = (_lib.StatsC * count)()
    status = np.zeros(count, dtype=np.int32)
    span = C.c_double()
    rc = getattr(_lib.lib(), entry)(ctxs, count, rp, xp, float(rtol), float(atol), int(max_cycles), comp,
                                    _PRECISION[precision], int(workers), stats, _lib.ptr(status, C.c_int32),
                                    C.byref(span))
    if rc != _lib.TPA_OK:
        bad = np.nonzero(status)[0]
        if len(bad) == 0:
            raise _lib.TpaError(int(rc), f"{entry}: invalid arguments")
        k = int(bad[0])
        msg = _lib.lib().tpa_last_error(solvers[k].ctx.handle).decode()
        raise _lib.TpaError(int(rc), f"{entry}: problem {k}: {msg}")
    out = BatchResult(s._stats_from(st) for s, st in zip(solvers, stats))
    out.device_ms = span.value
    return out


def solve(solution, solver, rhs, *, rtol=1e-10, atol=0.0, max_cycles=100, compatibility="project", precision=None):
    """`solve!(solution, solver, rhs)`: solve L(solution) = rhs in place.

    `rhs` is the strong-form right-hand side and `solution` the initial guess,
    both float64 arrays in cell order; `solution` is overwritten.  Returns the
    solver's `LinearSolverStats`.
    """
    if not 0 <= rtol < 1:
        raise ValueError("rtol must lie in [0, 1)")
    if atol < 0:
        raise ValueError("atol must be nonnegative")
    if max_cycles < 0:
        raise ValueError("max_cycles must be nonnegative")
    comp = _compat(compatibility)
    if not (isinstance(solution, np.ndarray) and solution.dtype == np.float64 and solution.flags.c_contiguous):
        raise TypeError("solution must be a contiguous float64 array")
    n = solver.operator.mesh.ncells
    if solution.shape != (n,) or np.shape(rhs) != (n,):
        raise ValueError("fields and multigrid solver must share a mesh")
    b = _lib.f64(rhs)
    st = _lib.StatsC()
    solver.ctx.call("tpa_solve", _lib.ptr(b, C.c_double), _lib.ptr(solution, C.c_double), float(rtol), float(atol),
                    int(max_cycles), comp, _PRECISION[precision or solver.precision], C.byref(st))
    return solver._stats_from(st)
