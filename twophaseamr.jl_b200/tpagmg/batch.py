"""Merged batch of independent pressure solves (`tpa_batch_*`).

The reference solves independent problems one `solve!` at a time, one
`EllipticSolver` per problem (src/solvers/multigrid/elliptic_solver.jl:628-675
of ronaldremmerswaal/TwoPhaseAMR.jl).  `BatchedSolver` merges the hierarchies
of many `EllipticSolver`s into one set of batch levels on the GPU, so that one
kernel launch advances a V-cycle phase of every problem; each problem keeps
its own CG scalars, stopping rules and statistics.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .solver import _PRECISION, _compat


class BatchedSolver:
    """Merged batch of the given solvers' problems (copied at construction)."""

    def __init__(self, solvers):
        if not solvers:
            raise ValueError("a batch needs at least one solver")
        self.solvers = list(solvers)
        ctxs = (C.c_void_p * len(self.solvers))(*[s.ctx.handle.value for s in self.solvers])
        self.handle = C.c_void_p()
        rc = _lib.lib().tpa_batch_create(C.byref(self.handle), ctxs, len(self.solvers))
        if rc != _lib.TPA_OK:
            msg = _lib.lib().tpa_batch_last_error(self.handle).decode() if self.handle else "tpa_batch_create"
            self.close()
            raise _lib.TpaError(rc, f"tpa_batch_create: {msg}")
        out = np.zeros(4, dtype=np.int64)
        self._call("tpa_batch_sizes", _lib.ptr(out, C.c_int64))
        self.count, self.ncells, self.levels, self.tail_levels = (int(v) for v in out)
        self.offsets = np.zeros(self.count + 1, dtype=np.int64)
        self._call("tpa_batch_offsets", _lib.ptr(self.offsets, C.c_int64))
        self.stats = []

    def _call(self, name, *args):
        rc = getattr(_lib.lib(), name)(self.handle, *args)
        if rc != _lib.TPA_OK:
            raise _lib.TpaError(rc, f"{name}: {_lib.lib().tpa_batch_last_error(self.handle).decode()}")

    def close(self):
        if self.handle:
            _lib.lib().tpa_batch_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def split(self, v):
        """Per-problem views of a concatenated cell array."""
        return [v[a:b] for a, b in zip(self.offsets[:-1], self.offsets[1:])]

    def concat(self, fields):
        if len(fields) != self.count:
            raise ValueError("one field per problem is required")
        out = np.concatenate([np.asarray(f, dtype=np.float64) for f in fields])
        if out.shape != (self.ncells,):
            raise ValueError("fields and batch must share meshes")
        return out

    def set_stream(self, stream):
        self._call("tpa_batch_set_stream", C.c_void_p(int(stream) or None))

    def _stats(self, raw):
        self.stats = []
        for s, st in zip(self.solvers, raw):
            s._stats_from(st)
            self.stats.append(dict(cycles=st.cycles, converged=bool(st.converged), initial_linf=st.initial_linf,
                                   final_linf=st.final_linf, target_linf=st.target_linf, restarts=st.restarts,
                                   removed_rhs_mean=st.removed_rhs_mean, device_ms=st.device_ms,
                                   kernel_launches=st.kernel_launches))
        return self.stats

    def solve(self, x, rhs, *, rtol=1e-10, atol=0.0, max_cycles=100, compatibility="project", precision="mixed"):
        """`solve!` of every problem.  x (initial guesses in, solutions out) and
        rhs are concatenated float64 host arrays (offsets: `self.offsets`)."""
        if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous
                and x.shape == (self.ncells,)):
            raise TypeError("x must be a contiguous float64 array of the batch's cells")
        b = _lib.f64(rhs)
        if b.shape != (self.ncells,):
            raise ValueError("rhs must hold the batch's cells")
        raw = (_lib.StatsC * self.count)()
        status = np.zeros(self.count, dtype=np.int32)
        self._call("tpa_batch_solve", _lib.ptr(b, C.c_double), _lib.ptr(x, C.c_double), float(rtol), float(atol),
                   int(max_cycles), _compat(compatibility), _PRECISION[precision], raw, _lib.ptr(status, C.c_int32))
        return self._stats(raw)

    def solve_device(self, rhs_ptr, x_ptr, *, rtol=1e-10, atol=0.0, max_cycles=100, compatibility="project",
                     precision="mixed"):
        """`solve` on concatenated device arrays (raw CUDA pointers)."""
        raw = (_lib.StatsC * self.count)()
        status = np.zeros(self.count, dtype=np.int32)
        self._call("tpa_batch_solve_device", C.c_void_p(rhs_ptr), C.c_void_p(x_ptr), float(rtol), float(atol),
                   int(max_cycles), _compat(compatibility), _PRECISION[precision], raw, _lib.ptr(status, C.c_int32))
        return self._stats(raw)
