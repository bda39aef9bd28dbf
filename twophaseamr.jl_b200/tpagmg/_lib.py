"""ctypes binding of `libtpagmg.so` (the C-ABI declared in include/tpagmg.h).

The library is loaded from `tpagmg/_lib/` inside the source tree.  There is no
CPU fallback: if the library is missing, importing the solver raises, and every
device entry point returns TPA_ERR_CUDA on a machine without a CUDA device.
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

LIB_PATH = pathlib.Path(__file__).resolve().parent / "_lib" / "libtpagmg.so"

TPA_OK = 0
TPA_ERR_INVALID_ARG = 1
TPA_ERR_CUDA = 2
TPA_ERR_TIMEOUT = 3
TPA_ERR_NONFINITE = 4
TPA_ERR_UNSUPPORTED = 5
TPA_ERR_STATE = 7


class TpaError(RuntimeError):
    """A failed library call; `code` is the tpa_status."""

    def __init__(self, code, message):
        super().__init__(f"[tpa_status {code}] {message}")
        self.code = code


class MultigridOptionsC(C.Structure):
    _fields_ = [("coarse_size", C.c_int32), ("pre_sweeps", C.c_int32),
                ("post_sweeps", C.c_int32), ("max_levels", C.c_int32), ("smoother", C.c_int32)]


class StatsC(C.Structure):
    _fields_ = [("cycles", C.c_int32), ("converged", C.c_int32), ("compatible", C.c_int32),
                ("restarts", C.c_int32), ("initial_l2", C.c_double), ("initial_linf", C.c_double),
                ("final_l2", C.c_double), ("final_linf", C.c_double), ("target_linf", C.c_double),
                ("residual_scale", C.c_double), ("removed_rhs_mean", C.c_double),
                ("device_ms", C.c_double), ("kernel_launches", C.c_int32), ("precision", C.c_int32),
                ("removed_rhs_max_component_mean", C.c_double)]


class TuneC(C.Structure):
    _fields_ = [("tail_cells", C.c_int32), ("tail_ctas", C.c_int32), ("structured", C.c_int32),
                ("vectorized", C.c_int32), ("pdl", C.c_int32), ("fuse_restrict", C.c_int32),
                ("persistent", C.c_int32), ("tiles", C.c_int32),
                ("ms_per_vcycle", C.c_double)]


class CmdgfmSystemC(C.Structure):
    _fields_ = [("np", C.c_int64), ("nx", C.c_int64), ("row_ptr", C.c_void_p), ("col", C.c_void_p),
                ("val", C.c_void_p), ("rhs", C.c_void_p), ("pressure_cell", C.c_void_p),
                ("pressure_anchor", C.c_void_p), ("defect_weight", C.c_void_p), ("na", C.c_int64),
                ("extra_row_ptr", C.c_void_p), ("extra_col", C.c_void_p), ("extra_val", C.c_void_p),
                ("extra_rhs", C.c_void_p), ("extra_weight", C.c_void_p), ("row_scale", C.c_void_p),
                ("col_scale", C.c_void_p), ("drop_tolerance", C.c_double), ("tolerance", C.c_double),
                ("max_iterations", C.c_int32), ("precision", C.c_int32), ("initial_pressure", C.c_void_p),
                ("warm_start", C.c_int32)]


class CmdgfmStatsC(C.Structure):
    _fields_ = [("converged", C.c_int32), ("iterations", C.c_int32), ("attempts", C.c_int32),
                ("kernel_launches", C.c_int32), ("initial_residual", C.c_double), ("final_residual", C.c_double),
                ("pressure_defect", C.c_double), ("jump_defect", C.c_double), ("anchor_defect", C.c_double),
                ("setup_ms", C.c_double), ("device_ms", C.c_double), ("factor_entries", C.c_int64),
                ("lower_levels", C.c_int32), ("upper_levels", C.c_int32), ("inverse_entries", C.c_int64),
                ("initial_guess_used", C.c_int32)]


P = C.c_void_p
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
f64p = C.POINTER(C.c_double)
i8p = C.POINTER(C.c_int8)

SIGNATURES = {
    "tpa_create": (C.c_int32, [C.POINTER(P), C.c_int32]),
    "tpa_destroy": (None, [P]),
    "tpa_last_error": (C.c_char_p, [P]),
    "tpa_set_mesh": (C.c_int32, [P, i32p, i32p, i32p, f64p, f64p, C.c_int64, i32p]),
    "tpa_mesh_sizes": (C.c_int32, [P, i64p]),
    "tpa_mesh_blocks": (C.c_int32, [P, i32p, f64p]),
    "tpa_mesh_faces": (C.c_int32, [P, i32p, i32p, i8p, f64p]),
    "tpa_mesh_boundary_faces": (C.c_int32, [P, i32p, i8p, i8p, f64p]),
    "tpa_set_operator": (C.c_int32, [P, f64p]),
    "tpa_set_open_boundaries": (C.c_int32, [P, i32p, f64p]),
    "tpa_metric_offdiagonal_count": (C.c_int32, [P, i64p]),
    "tpa_build_hierarchy": (C.c_int32, [P, C.POINTER(MultigridOptionsC)]),
    "tpa_hierarchy_sizes": (C.c_int32, [P, i32p, i64p, C.c_int32]),
    "tpa_level_owners": (C.c_int32, [P, C.c_int32, i32p]),
    "tpa_level_info": (C.c_int32, [P, C.c_int32, f64p, f64p, i32p]),
    "tpa_level_face_coefficients": (C.c_int32, [P, C.c_int32, f64p]),
    "tpa_refresh": (C.c_int32, [P, f64p]),
    "tpa_last_refresh": (C.c_int32, [P, i32p, f64p]),
    "tpa_solve": (C.c_int32, [P, f64p, f64p, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_int32,
                              C.POINTER(StatsC)]),
    "tpa_solve_device": (C.c_int32, [P, P, P, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_int32,
                                     C.POINTER(StatsC)]),
    "tpa_solve_batched": (C.c_int32, [C.POINTER(P), C.c_int32, C.POINTER(f64p), C.POINTER(f64p), C.c_double,
                                      C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(StatsC),
                                      i32p, f64p]),
    "tpa_solve_batched_device": (C.c_int32, [C.POINTER(P), C.c_int32, C.POINTER(P), C.POINTER(P), C.c_double,
                                             C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                             C.POINTER(StatsC), i32p, f64p]),
    "tpa_autotune": (C.c_int32, [P, C.c_int32, C.c_int32, C.POINTER(TuneC), C.POINTER(TuneC), C.c_int32, i32p]),
    "tpa_set_tuning": (C.c_int32, [P, C.POINTER(TuneC)]),
    "tpa_get_tuning": (C.c_int32, [P, C.POINTER(TuneC)]),
    "tpa_batch_create": (C.c_int32, [C.POINTER(P), C.POINTER(P), C.c_int32]),
    "tpa_batch_destroy": (None, [P]),
    "tpa_batch_last_error": (C.c_char_p, [P]),
    "tpa_batch_sizes": (C.c_int32, [P, i64p]),
    "tpa_batch_offsets": (C.c_int32, [P, i64p]),
    "tpa_batch_set_stream": (C.c_int32, [P, P]),
    "tpa_batch_solve": (C.c_int32, [P, f64p, f64p, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_int32,
                                    C.POINTER(StatsC), i32p]),
    "tpa_batch_solve_device": (C.c_int32, [P, P, P, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_int32,
                                           C.POINTER(StatsC), i32p]),
    "tpa_adjoint": (C.c_int32, [P, f64p, f64p, f64p, f64p, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                C.POINTER(StatsC)]),
    "tpa_adjoint_device": (C.c_int32, [P, P, P, P, P, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                       C.POINTER(StatsC)]),
    "tpa_face_coefficient_gradient": (C.c_int32, [P, f64p, f64p, f64p]),
    "tpa_apply": (C.c_int32, [P, f64p, f64p]),
    "tpa_vcycle": (C.c_int32, [P, f64p, f64p, C.c_int32]),
    "tpa_synchronize": (C.c_int32, [P]),
    "tpa_set_stream": (C.c_int32, [P, P]),
    "tpa_device_info": (C.c_int32, [P, i64p]),
    "tpa_tiled_levels": (C.c_int32, [P, i32p]),
    "tpa_streamed_levels": (C.c_int32, [P, i32p]),
    "tpa_residual_norms": (C.c_int32, [P, P, f64p]),
    "tpa_residual_norms_noalloc": (C.c_int32, [P, P, P, C.c_int64, f64p]),
    "tpa_time_kernel": (C.c_int32, [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, f64p]),
    "tpa_refresh_device": (C.c_int32, [P, P]),
    "tpa_level_red_black": (C.c_int32, [P, C.c_int32, C.POINTER(C.c_uint8), f64p]),
    "tpa_conditional_fraction_device": (C.c_int32, [P, P, C.c_double, P, P]),
    "tpa_face_coefficients_device": (C.c_int32, [P, P, C.c_double, C.c_double, P]),
    "tpa_surface_tension_device": (C.c_int32, [P, P, C.c_double, C.c_double, C.c_int32, P, P]),
    "tpa_weighted_gradient_device": (C.c_int32, [P, P, P, P]),
    "tpa_divergence_device": (C.c_int32, [P, P, P, P]),
    "tpa_project": (C.c_int32, [P, f64p, f64p, f64p, P, C.POINTER(StatsC)]),
    "tpa_project_device": (C.c_int32, [P, P, P, P, P, C.POINTER(StatsC)]),
    "tpa_level_matrix": (C.c_int32, [P, C.c_int32, i64p, i64p, i32p, f64p]),
    "tpa_cmdgfm_solve": (C.c_int32, [P, C.POINTER(CmdgfmSystemC), f64p, C.POINTER(CmdgfmStatsC)]),
    "tpa_cmdgfm_factor": (C.c_int32, [C.POINTER(CmdgfmSystemC), i64p, i64p, i32p, f64p, i64p, i64p, i32p, f64p,
                                      i64p, i64p, i32p, f64p]),
}

_lib = None


def lib():
    """Load the library once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"libtpagmg.so not built: run `python twophaseamr.jl_b200/build.py` ({LIB_PATH})")
        handle = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None


class Context:
    """Owns one `tpa_context`."""

    def __init__(self, device=0):
        self.handle = P()
        self._check(lib().tpa_create(C.byref(self.handle), int(device)), "tpa_create")

    def _check(self, status, what):
        if status != TPA_OK:
            msg = lib().tpa_last_error(self.handle).decode() if self.handle else what
            raise TpaError(status, f"{what}: {msg}")

    def call(self, name, *args):
        self._check(getattr(lib(), name)(self.handle, *args), name)

    def close(self):
        if self.handle:
            lib().tpa_destroy(self.handle)
            self.handle = P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)
