"""Oracle (test infrastructure only): ctypes driver of `cgmg.c`, the C/OpenMP
restatement of the reference's V-cycle + CG loop, and the timed CPU baseline.

`build()` compiles `oracle/_build/libcgmg.so` with gcc; `Runner` packs a Python
oracle hierarchy (oracle.multigrid) for the C code; `bench_droplet` times the
droplet workload the B200 bench uses.
"""
from __future__ import annotations

import ctypes as C
import os
import pathlib
import subprocess
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB = HERE / "_build" / "libcgmg.so"


def build():
    LIB.parent.mkdir(exist_ok=True)
    src = HERE / "cgmg.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.check_call(["gcc", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=c11",
                               str(src), "-o", str(LIB), "-lm"])
    return LIB


i64p, i32p, f64p, i8p = C.POINTER(C.c_int64), C.POINTER(C.c_int32), C.POINTER(C.c_double), C.POINTER(C.c_int8)


class Level(C.Structure):
    _fields_ = [("n", C.c_int64), ("rp", i64p), ("ci", i32p), ("v", f64p), ("dinv", f64p), ("w", C.c_double),
                ("vol", f64p), ("slot", i32p), ("ncomp", C.c_int32), ("cvol", f64p),
                ("prp", i64p), ("pci", i32p), ("pv", f64p), ("trp", i64p), ("tci", i32p), ("tv", f64p),
                ("x", f64p), ("b", f64p), ("t", f64p), ("r", f64p)]


class Fine(C.Structure):
    _fields_ = [("nc", C.c_int64), ("nf", C.c_int64), ("fm", i32p), ("fp", i32p), ("area", f64p), ("sk", f64p),
                ("kp", i64p), ("ki", i32p), ("kv", f64p), ("inc_off", i64p), ("inc_face", i32p), ("inc_sign", i8p),
                ("fin", f64p), ("fout", f64p)]


class Stats(C.Structure):
    _fields_ = [("cycles", C.c_int32), ("converged", C.c_int32), ("initial_linf", C.c_double),
                ("final_linf", C.c_double), ("target", C.c_double)]


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


class Runner:
    """Holds a packed copy of a Python oracle hierarchy for `cgmg_solve`."""

    def __init__(self, op, mg):
        self.lib = C.CDLL(str(build()))
        self.lib.cgmg_solve.restype = C.c_int
        self.keep = []
        k = lambda a, dt: self.keep.append(np.ascontiguousarray(a, dtype=dt)) or self.keep[-1]
        levels = (Level * len(mg.levels))()
        for l, lev in enumerate(mg.levels):
            A = lev.matrix.tocsr()
            A.sort_indices()
            L = levels[l]
            L.n = lev.n
            L.rp, L.ci, L.v = _p(k(A.indptr, np.int64), C.c_int64), _p(k(A.indices, np.int32), C.c_int32), \
                _p(k(A.data, np.float64), C.c_double)
            L.dinv = _p(k(lev.inverse_diagonal, np.float64), C.c_double)
            L.w = lev.weight
            L.vol = _p(k(lev.volumes, np.float64), C.c_double)
            slots = lev.slots if lev.singular else np.full(lev.n, -1)
            L.slot = _p(k(slots, np.int32), C.c_int32)
            L.ncomp = len(lev.component_volumes)
            L.cvol = _p(k(lev.component_volumes if lev.singular else np.zeros(1), np.float64), C.c_double)
            if lev.prolongation is not None:
                P = lev.prolongation.tocsr()
                P.sort_indices()
                T = lev.prolongation.T.tocsr()
                T.sort_indices()
                L.prp, L.pci, L.pv = _p(k(P.indptr, np.int64), C.c_int64), _p(k(P.indices, np.int32), C.c_int32), \
                    _p(k(P.data, np.float64), C.c_double)
                L.trp, L.tci, L.tv = _p(k(T.indptr, np.int64), C.c_int64), _p(k(T.indices, np.int32), C.c_int32), \
                    _p(k(T.data, np.float64), C.c_double)
            for name in ("x", "b", "t", "r"):
                setattr(L, name, _p(k(np.zeros(lev.n), np.float64), C.c_double))
        self.levels = levels
        mesh = op.mesh
        F = Fine()
        F.nc, F.nf = mesh.ncells, mesh.nfaces
        F.fm, F.fp = _p(k(mesh.face_minus, np.int32), C.c_int32), _p(k(mesh.face_plus, np.int32), C.c_int32)
        F.area, F.sk = _p(k(mesh.face_area, np.float64), C.c_double), _p(k(op.sqrt_kappa, np.float64), C.c_double)
        Kr = op.K.tocsr()
        Kr.sort_indices()
        F.kp, F.ki, F.kv = _p(k(Kr.indptr, np.int64), C.c_int64), _p(k(Kr.indices, np.int32), C.c_int32), \
            _p(k(Kr.data, np.float64), C.c_double)
        nf = mesh.nfaces
        cells = np.concatenate([mesh.face_minus, mesh.face_plus])
        faces = np.concatenate([np.arange(nf), np.arange(nf)])
        signs = np.concatenate([-np.ones(nf), np.ones(nf)])
        order = np.lexsort((faces, cells))
        off = np.concatenate([[0], np.cumsum(np.bincount(cells, minlength=mesh.ncells))])
        F.inc_off = _p(k(off, np.int64), C.c_int64)
        F.inc_face = _p(k(faces[order], np.int32), C.c_int32)
        F.inc_sign = _p(k(signs[order], np.int8), C.c_int8)
        F.fin, F.fout = _p(k(np.zeros(nf), np.float64), C.c_double), _p(k(np.zeros(nf), np.float64), C.c_double)
        self.fine = F
        c = mg.levels[-1]
        A = mg.coarse_matrix.toarray()
        inv = np.linalg.inv(A)[: c.n, : c.n]
        self.cinv = k(inv, np.float64)
        self.cn = c.n
        self.pre, self.post = mg.pre_sweeps, mg.post_sweeps

    def solve(self, rhs, x0=None, rtol=1e-10, atol=0.0, max_cycles=100, threads=0):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.zeros(len(rhs)) if x0 is None else np.array(x0, dtype=np.float64)
        st = Stats()
        self.lib.cgmg_solve(C.c_int(len(self.levels)), self.levels, C.byref(self.fine), _p(self.cinv, C.c_double),
                            C.c_int64(self.cn), C.c_int(self.pre), C.c_int(self.post), _p(rhs, C.c_double),
                            _p(x, C.c_double), C.c_double(rtol), C.c_double(atol), C.c_int(max_cycles),
                            C.c_int(threads), C.byref(st))
        return x, st


def droplet_problem(levels=4):
    """The bench's droplet workload built with the oracle alone."""
    import sys
    sys.path.insert(0, str(HERE.parent / "twophaseamr.jl_b200"))
    from tpagmg import workloads as W
    from tpagmg.operator import mixture_density
    from .mesh import block_tree_mesh
    from .multigrid import MultigridOptions, TreeGeometricMultigrid
    from .operator import PoissonOperator

    # the oracle mesh carries the attributes the input generators read
    mesh = block_tree_mesh(**W.droplet_spec(levels=levels))
    frac = W.circle_fractions(mesh)
    kappa = 1.0 / mixture_density(mesh, frac, (1000.0, 1.0))
    psi = 0.072 / 0.15 * (frac > 0.5)
    op = PoissonOperator(mesh, kappa)
    mg = TreeGeometricMultigrid(op, MultigridOptions())
    rhs = W.droplet_rhs(mesh, op.apply(psi))
    return mesh, op, mg, rhs


def bench_droplet(steps=10, warmup=3, levels=4, threads=None, problem=None):
    """Time `steps` warm solves of the droplet workload (after `warmup`
    untimed ones) with `threads` OpenMP threads; ms_per_step is their median.
    `problem` is an already built `droplet_problem(levels)`."""
    threads = threads or os.cpu_count()
    mesh, op, mg, rhs = problem or droplet_problem(levels)
    run = Runner(op, mg)
    for _ in range(warmup):
        run.solve(rhs, threads=threads)
    ts, its = [], []
    for _ in range(max(1, steps)):
        t0 = time.perf_counter()
        x, st = run.solve(rhs, threads=threads)
        ts.append(time.perf_counter() - t0)
        its.append(st.cycles)
        assert st.converged
    ms = 1e3 * float(np.median(ts))
    return {"cells": mesh.ncells, "iterations": float(np.median(its)), "ms_per_step": ms, "threads": threads,
            "cell_updates_per_s": mesh.ncells * float(np.median(its)) / (ms * 1e-3), "runner": run}
