"""Benchmark of the B200 pressure solve (one JSON line on rank 0).

Workload: the two-phase droplet pressure solve on an adaptive tree (unit
square, free-slip walls, 4x4 blocks of 16x16 cells refined 4 levels to
h = 1/1024 in a band of 8 finest cells around the circle |x - (0.5, 0.6)| =
0.15; density 1000 inside, 1 outside; CGFM surface-tension RHS plus N(0, 1)
noise), solved to relative residual 1e-10 (strong L-infinity, the reference's
`solve!(...; rtol=1e-10)`).  A step is one complete solve.

metric: cell-updates/s = fine cells x CG iterations / time, for the mixed
precision (FP32 V-cycle inside FP64 CG) solve; the FP64 solve on the same mesh
is reported beside it.  Inputs are resident in HBM for `value`; `e2e` goes
through the public C-ABI (`tpa_solve`) with pinned host buffers, host<->device
copies inside the timed region.  The L2 is flushed (a 256 MiB write) between
timed steps because the working set (~20 MB) fits in L2.

`--impl reference` times the CPU restatement of the reference solve (the
reference is Julia and does not run here) on the same workload.
"""
import argparse
import json
import os
import pathlib
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path[:0] = [str(ROOT), str(ROOT / "twophaseamr.jl_b200")]

RTOL = 1e-10
HBM_FALLBACK = 6650.0
# one metric string for both arms (the precision is carried by `dtype`)
DROPLET_METRIC = "cell-updates/s to rel. residual 1e-10 (droplet AMR pressure solve)"


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK, "fallback"


def workload(levels=4):
    from tpagmg import workloads as W
    return W.droplet_spec(levels=levels)


def rank_share(items, rank, world):
    """The independent problems one rank solves (round robin; no data exchange)."""
    return list(items)[rank::world]


def combine_over_ranks(max_vals, sum_vals, world, device="cpu"):
    """Max over ranks of the timings and sum of the work counts (the only
    collectives of the multi-rank bench: every rank calls it once, in the same
    order)."""
    import torch
    import torch.distributed as dist
    mx = torch.tensor([float(v) for v in max_vals], dtype=torch.float64, device=device)
    sm = torch.tensor([float(v) for v in sum_vals], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return [float(v) for v in mx.cpu()], [float(v) for v in sm.cpu()]


def reference_arm(args):
    """CPU restatement of the reference solve, on this host's cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import cgmg
    res = cgmg.bench_droplet(steps=args.steps, warmup=args.warmup, levels=args.levels)
    line = {
        "impl": "reference", "metric": DROPLET_METRIC,
        "value": res["cell_updates_per_s"], "unit": "cell-updates/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": res["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Philox)",
        "config": {"workload": f"droplet_amr levels={args.levels}", "fine_cells": res["cells"],
                   "cg_iterations": res["iterations"], "threads": res["threads"]},
        "cpu_baseline": {"value": res["cell_updates_per_s"], "unit": "cell-updates/s", "cores": res["threads"],
                         "kind": "port",
                         "sample": f"median of {args.steps} warm full solves of the droplet workload "
                                   f"({args.warmup} untimed), {res['threads']} OpenMP threads"},
        "e2e": {"value": res["cell_updates_per_s"], "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def model_bytes_per_cell_iteration(s, s_kappa):
    """Compulsory HBM bytes per fine cell and CG iteration of the solve: a
    V-cycle (hierarchy factor 4/3; two pre-sweeps reading x, b and two face
    coefficients and writing x; residual + restriction; prolongation +
    correction) in value size s with coefficient size s_kappa (0 when
    constant), plus 56 bytes of the FP64 CG (operator product and the fused
    vector updates)."""
    vcycle = 4.0 / 3.0 * (4 * (3 * s + 2 * s_kappa) + (2 * s + 2 * s_kappa + s / 4) + (2 * s + s / 4))
    return vcycle + 56.0


def whole_solve_roofline(n, variable_kappa, mixed, fp64, peak, peak_kind, world=1):
    """Model bytes of whole solves (per-iteration model times iterations) over
    their measured time, against the measured HBM bandwidth."""
    out = {"peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
           "what": "model bytes per cell and CG iteration x cells x iterations / solve time"}
    for name, (its, ms), s in (("mixed", mixed, 4), ("fp64", fp64, 8)):
        b = model_bytes_per_cell_iteration(s, s if variable_kappa else 0)
        gbs = world * n * its * b / (ms * 1e-3) / 1e9
        out[name] = {"bytes_per_cell_iteration": b, "achieved": gbs, "frac": gbs / peak}
    return out


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = pathlib.Path(tempfile.gettempdir()) / f"tpagmg_clocks_{os.getpid()}.csv"

    def __enter__(self):
        self.t0 = time.perf_counter()
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            # nvidia-smi needs about a second to emit its first samples
            left = 1.5 - (time.perf_counter() - self.t0)
            if left > 0:
                time.sleep(left)
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in self.path.read_text().strip().splitlines() if r.strip()]
            sm = [float(r[0]) for r in rows]
            reasons = set()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for r in rows:
                for k, n in enumerate(names):
                    if "Active" in r[3 + k] and "Not" not in r[3 + k]:
                        reasons.add(n)
            return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(rows[0][1]), "reasons": sorted(reasons),
                    "samples": len(rows)}
        except Exception as e:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "error": str(e)}


def batch_main(args):
    """Batched uneven solves: `--batch` independent two-phase problems (tree
    depth 2..6, circle radius U[0.05, 0.3], density ratio 10/100/1000), each
    solved to rel. residual 1e-10 in mixed precision; a step is one batched
    solve of every problem.  Ranks split the problem list (no communication)."""
    from concurrent.futures import ThreadPoolExecutor
    import torch
    import torch.distributed as dist
    from tpagmg import BatchedSolver, EllipticSolver, PoissonOperator, BlockTreeMesh, solve_batched
    from tpagmg import workloads as W

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=300))
    problems = rank_share(W.batch_problems(args.batch), rank, world)
    t0 = time.perf_counter()

    def make(p):
        m = BlockTreeMesh(**W.batch_spec(p))
        kappa, rhs = W.batch_inputs(m, p)
        return m, EllipticSolver(PoissonOperator(m, kappa), device=local), rhs

    with ThreadPoolExecutor(max(1, min(32, os.cpu_count() or 1))) as ex:
        built = list(ex.map(make, problems))
    setup_s = time.perf_counter() - t0
    solvers = [s for _, s, _ in built]
    sizes = [m.ncells for m, _, _ in built]
    offs = np.concatenate([[0], np.cumsum(sizes)])
    rhs_all = torch.from_numpy(np.concatenate([r for _, _, r in built])).cuda()
    x_all = torch.zeros(int(offs[-1]), dtype=torch.float64, device="cuda")
    rptr = [rhs_all.data_ptr() + 8 * int(o) for o in offs[:-1]]
    xptr = [x_all.data_ptr() + 8 * int(o) for o in offs[:-1]]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def step_streams(precision):
        x_all.zero_()
        torch.cuda.synchronize()
        res = solve_batched(xptr, solvers, rptr, rtol=RTOL, precision=precision, workers=args.workers)
        assert all(st.converged for st in res)
        its = [st.cycles for st in res]
        return res.device_ms, its, sum(st.kernel_launches for st in res)

    t0 = time.perf_counter()
    merged = BatchedSolver(solvers) if args.batch_mode == "merged" else None
    merge_s = time.perf_counter() - t0

    def step_merged(precision):
        x_all.zero_()
        torch.cuda.synchronize()
        st = merged.solve_device(rhs_all.data_ptr(), x_all.data_ptr(), rtol=RTOL, precision=precision)
        assert all(s["converged"] for s in st)
        return st[0]["device_ms"], [s["cycles"] for s in st], st[0]["kernel_launches"]

    step = step_merged if merged else step_streams
    if args.profile:
        # only W warm-up and K mixed solves of the batch (for ncu launch lists)
        launches = 0
        for _ in range(args.warmup + args.steps):
            launches += step("mixed")[2]
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"profile": f"batch_{args.batch} mixed", "solves": args.steps,
                              "kernel_launches": launches}))
        return 0
    streams_ms = None
    if merged:
        # the per-problem-stream path on the same problems, for comparison
        step_streams("mixed")
        streams_ms = step_streams("mixed")[0]

    for _ in range(args.warmup):
        step("mixed")
        step("fp64")
    if world > 1:
        dist.barrier()
    clk = ClockSampler(local).__enter__()

    def timed(precision):
        ms, upd, launches = [], [], 0
        for _ in range(args.steps):
            flush.fill_(1.0)
            span, its, nl = step(precision)
            ms.append(span)
            upd.append(float(np.dot(sizes, its)))
            launches += nl
        return float(np.mean(ms)), float(np.mean(upd)), launches

    mixed_ms, mixed_upd, launches = timed("mixed")
    fp64_ms, fp64_upd, _ = timed("fp64")
    clk.__exit__(None, None, None)
    # errors of the mixed solutions against the FP64 ones, per problem
    step("fp64")
    x64 = x_all.clone()
    step("mixed")
    errs = [float((x_all[a:b] - x64[a:b]).abs().max() / x64[a:b].abs().max()) for a, b in zip(offs[:-1], offs[1:])]
    # end to end: pinned host arrays through the public batched entry point,
    # copies inside
    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).pin_memory()
        return t, t.numpy()
    keep = [pinned(np.zeros(n)) for n in sizes] + [pinned(r) for _, _, r in built]
    xs = [a for _, a in keep[:len(sizes)]]
    rh = [a for _, a in keep[len(sizes):]]
    xcat_t, xcat = pinned(np.zeros(int(offs[-1])))
    rcat_t, rcat = pinned(np.concatenate([r for _, _, r in built]))
    e2e = []
    for k in range(args.steps + 1):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        if merged:
            xcat[:] = 0
            res = merged.solve(xcat, rcat, rtol=RTOL, precision="mixed")
            its = [s["cycles"] for s in res]
        else:
            for x in xs:
                x[:] = 0
            res = solve_batched(xs, solvers, rh, rtol=RTOL, precision="mixed", workers=args.workers)
            its = [st.cycles for st in res]
        if k:
            e2e.append((time.perf_counter() - t1) * 1e3)
    e2e_upd = float(np.dot(sizes, its))
    (mixed_ms, fp64_ms, e2e_ms), (mixed_upd, fp64_upd, e2e_upd, cells) = combine_over_ranks(
        [mixed_ms, fp64_ms, float(np.mean(e2e))], [mixed_upd, fp64_upd, e2e_upd, float(sum(sizes))], world, "cuda")
    peak, peak_kind = measured_peaks()
    # algorithmic bytes per fine cell and CG iteration (FP32 V-cycle with variable
    # coefficients, hierarchy factor 4/3, plus the FP64 CG vectors)
    b_cell = 4.0 / 3.0 * (4 * (3 * 4 + 2 * 4) + (2 * 4 + 2 * 4 + 1) + (2 * 4 + 1)) + 56.0
    achieved = mixed_upd * b_cell / (mixed_ms * 1e-3) / 1e9
    line = {
        "metric": f"cell-updates/s to rel. residual 1e-10 ({args.batch} batched uneven two-phase solves, mixed)",
        "value": mixed_upd / (mixed_ms * 1e-3), "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mixed_ms, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic (seeded Philox)",
        "config": {"workload": f"batch_{args.batch} (base 2x2 roots of 16x16, depth U{{2..6}}, circle band)",
                   "problems": args.batch, "fine_cells_total": cells, "batch_mode": args.batch_mode,
                   "parallelism": f"problems split over {world} ranks" if world > 1 else "1 GPU",
                   "l2": "flushed between steps (256 MiB write)", "setup_s_rank0": setup_s,
                   "merge_s_rank0": merge_s,
                   "batch_levels": merged.levels if merged else None,
                   "tail_levels": merged.tail_levels if merged else None},
        "per_problem_streams_ms_per_step": streams_ms,
        "time_to_tolerance_ms": {"mixed": mixed_ms, "fp64": fp64_ms, "speedup_mixed_over_fp64": fp64_ms / mixed_ms},
        "fp64_value": fp64_upd / (fp64_ms * 1e-3),
        "mixed_error_vs_fp64_max": max(errs),
        "e2e": {"value": e2e_upd / (e2e_ms * 1e-3), "unit": "cell-updates/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": int(2 * 8 * cells), "d2h_bytes_per_step": int(8 * cells)},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "whole batched solve (model bytes per cell and CG iteration)",
                     "bytes_per_cell_iteration": b_cell, "peak_kind": peak_kind},
        "clocks": clk.summary(),
        "cpu_baseline": None,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def cmdgfm_measure(level, steps, warmup, profile=False, cpu=True):
    """The CMDGFM two-block solve (tpa_cmdgfm_solve) on the synthetic
    capillary-wave system of `level` refinement levels: median wall and device
    time of `steps` solves after `warmup`, with the FP32 V-cycle in the
    pressure block; beside it, the oracle's restatement (numpy/SciPy, one
    thread) on the same system when `cpu`."""
    import time as _t
    from tpagmg import BlockTreeMesh, EllipticSolver, PoissonOperator
    from tpagmg import workloads as W
    from tpagmg.cmdgfm import solve_cmdgfm
    from tpagmg.operator import mixture_density
    spec = W.capillary_wave_spec(level)
    m = BlockTreeMesh(**spec)
    fr = W.wave_fractions(m)
    kappa = 1.0 / mixture_density(m, fr, (1.0, 1e-3))
    s = EllipticSolver(PoissonOperator(m, kappa))
    if not profile:
        s.autotune(precision="mixed", vcycles=20)  # the pressure block's V-cycle layout
    system, exact = W.cmdgfm_system(m, s.level_matrix(0), kappa, fr)
    for _ in range(warmup):
        solve_cmdgfm(s, system, precision="mixed")
    wall, dev, st, x = [], [], None, None
    for _ in range(steps):
        t0 = _t.perf_counter()
        x, st = solve_cmdgfm(s, system, precision="mixed")
        wall.append((_t.perf_counter() - t0) * 1e3)
        dev.append(st.device_ms)
    if profile:
        return {"profile": f"cmdgfm capillary_wave L{level}", "solves": steps}
    npr = system.np_
    err = max(float(np.max(np.abs(x[:npr] - exact[:npr])) / np.max(np.abs(exact[:npr]))),
              float(np.max(np.abs(x[npr:] - exact[npr:])) / np.max(np.abs(exact[npr:]))))
    out = {"workload": f"capillary_wave L{level} (examples/07_capillary_wave mesh, {m.ncells} cells), "
                       f"synthetic CMDGFM system: {system.np_} pressures + {system.nx} jumps",
           "iterations": st.iterations, "converged": st.converged,
           "wall_ms": float(np.median(wall)), "device_ms": float(np.median(dev)), "setup_ms": st.setup_ms,
           "kernel_launches": st.kernel_launches, "factor_levels": [st.lower_levels, st.upper_levels],
           "error_vs_exact": err,
           "what": "tpa_cmdgfm_solve: residual replacement around BiCGSTAB with the FP32 GMG V-cycle on the reduced "
                   "pressure block and the Crout ILU of J - C D^-1 B on the jump block; host arrays in and out"}
    if cpu:
        import scipy.sparse as sp
        from oracle import cmdgfm as O  # the checker, timed as the CPU port
        from oracle.mesh import block_tree_mesh
        from oracle.multigrid import MultigridOptions, TreeGeometricMultigrid
        from oracle.operator import PoissonOperator as OOp
        M = sp.csr_matrix((system.val, system.col, system.row_ptr), shape=(system.n, system.n))
        E = sp.csr_matrix((system.extra_val, system.extra_col, system.extra_row_ptr), shape=(1, system.n))
        osys = O.CMDGFMSystem(matrix=M, rhs=system.rhs, np_=npr, pressure_cell=system.pressure_cell,
                              pressure_anchor=system.pressure_anchor, defect_weight=system.defect_weight, extra=E,
                              extra_rhs=system.extra_rhs, extra_weight=system.extra_weight,
                              row_scale=system.row_scale, col_scale=system.col_scale)
        mg = TreeGeometricMultigrid(OOp(block_tree_mesh(**spec), kappa), MultigridOptions())
        times = []
        for _ in range(3):
            t0 = _t.perf_counter()
            _, ost = O.solve(osys, mg)
            times.append((_t.perf_counter() - t0) * 1e3)
        out["cpu_port"] = {"ms": float(np.median(times)), "iterations": ost.iterations, "cores": 1,
                           "kind": "port", "sample": "median of 3 solves of the same system by the oracle "
                                                     "(numpy/SciPy restatement, hierarchy built once)"}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--levels", type=int, default=4)
    ap.add_argument("--workload", default="droplet_amr", choices=["droplet_amr", "uniform_2048", "batch", "cmdgfm"])
    ap.add_argument("--cmdgfm-level", type=int, default=6, help="refinement levels of the capillary-wave CMDGFM system")
    ap.add_argument("--batch", type=int, default=256, help="problems of the batch workload")
    ap.add_argument("--workers", type=int, default=32, help="host threads of the per-problem-stream batch")
    ap.add_argument("--batch-mode", default="merged", choices=["merged", "streams"],
                    help="merged batch levels (one launch per phase) or one stream per problem")
    ap.add_argument("--size", type=int, default=2048, help="cells per side of the uniform workload")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default device layout")
    ap.add_argument("--profile", action="store_true", help="only W warm-up and K solves (for ncu)")
    ap.add_argument("--profile-precision", default="mixed", choices=["mixed", "fp64", "mixed_ir"],
                    help="precision of the --profile solves")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "batch":
        return batch_main(args)
    if args.workload == "cmdgfm":
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        res = cmdgfm_measure(args.cmdgfm_level, args.steps, args.warmup, profile=args.profile,
                             cpu=not args.no_cpu_baseline)
        if not args.profile:
            res = {"metric": f"CMDGFM two-block solve time (capillary wave L{args.cmdgfm_level})",
                   "value": res["wall_ms"], "unit": "ms", "higher_is_better": False, "n_gpus": 1,
                   "steps": args.steps, "warmup": args.warmup, **res}
        print(json.dumps(res), flush=True)
        return

    import ctypes as C
    import torch
    import torch.distributed as dist
    from tpagmg import EllipticSolver, PoissonOperator, BlockTreeMesh
    from tpagmg import workloads as W
    from tpagmg import _lib

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    if args.workload == "droplet_amr":
        spec = workload(args.levels)
        mesh = BlockTreeMesh(**spec)
        frac, kappa, psi = W.droplet_inputs(mesh)
    else:  # uniform_2048: 128x128 periodic roots of 16x16, kappa = 1
        mesh = BlockTreeMesh(**W.uniform_spec(args.size))
        kappa = np.ones(mesh.nfaces)
    solver = EllipticSolver(PoissonOperator(mesh, kappa), device=local)
    stream = torch.cuda.current_stream()
    solver.ctx.call("tpa_set_stream", C.c_void_p(stream.cuda_stream))
    # each precision runs on the layout the autotuner found fastest for its own
    # V-cycle (the refinement solve runs the FP32 cycle: the mixed layout)
    layout, tune_s, layouts = solver.tuning(), 0.0, {}
    if not (args.no_autotune or args.profile):
        t0 = time.perf_counter()
        layouts["fp64"], _ = solver.autotune(precision="fp64", vcycles=20)
        layouts["mixed"], _ = solver.autotune(precision="mixed", vcycles=20)
        layout = layouts["mixed"]
        tune_s = time.perf_counter() - t0

    def use_layout(precision):
        lay = layouts.get("fp64" if precision == "fp64" else "mixed")
        if lay is not None:
            solver.set_tuning(**{k: v for k, v in lay.items() if k != "ms_per_vcycle"})
    if args.workload == "droplet_amr":
        rhs_h = W.droplet_rhs(mesh, solver.apply(psi))
    else:
        rhs_h = W.gaussian_rhs(mesh, W.SEEDS["uniform_2048"])
    n = mesh.ncells
    rhs_d = torch.from_numpy(rhs_h).cuda()
    x_d = torch.zeros(n, dtype=torch.float64, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > 126 MB L2

    def device_solve(precision):
        x_d.zero_()
        return solver.solve_device(rhs_d.data_ptr(), x_d.data_ptr(), rtol=RTOL, precision=precision)

    if args.profile:
        # profiling pass: W warm-up solves, then K solves and nothing else
        prec = args.profile_precision
        for _ in range(args.warmup):
            device_solve(prec)
        torch.cuda.synchronize()
        launches = 0
        for _ in range(args.steps):
            launches += device_solve(prec).kernel_launches
        torch.cuda.synchronize()
        print(json.dumps({"profile": f"{args.workload} {prec}", "solves": args.steps, "kernel_launches": launches}))
        return

    def timed(precision, steps):
        ms, its, launches = [], [], 0
        for _ in range(steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = device_solve(precision)
            e1.record(stream)
            e1.synchronize()
            assert st.converged, st
            ms.append(e0.elapsed_time(e1))
            its.append(st.cycles)
            launches += st.kernel_launches
        return float(np.mean(ms)), float(np.mean(its)), launches, ms

    # each precision on its layout: W warm-up solves, then K timed ones
    clk = ClockSampler(local).__enter__()
    res = {}
    for precision in ("mixed", "fp64", "mixed_ir"):
        use_layout(precision)
        for _ in range(args.warmup):
            device_solve(precision)
        barrier()
        res[precision] = timed(precision, args.steps)
    clk.__exit__(None, None, None)
    mixed_ms, mixed_it, mixed_launches, _ = res["mixed"]
    fp64_ms, fp64_it, _, _ = res["fp64"]
    ir_ms, ir_it, _, _ = res["mixed_ir"]
    use_layout("fp64")
    device_solve("fp64")
    x_ref = x_d.clone()
    use_layout("mixed")  # left in effect for the measurements below
    device_solve("mixed_ir")
    x_ir = x_d.clone()
    device_solve("mixed")
    x_mixed = x_d.clone()
    mixed_err = float((x_mixed - x_ref).abs().max() / x_ref.abs().max())
    ir_err = float((x_ir - x_ref).abs().max() / x_ref.abs().max())

    # max over ranks (each rank solves its own replica: no work to sum)
    (mixed_ms, fp64_ms, ir_ms), _ = combine_over_ranks([mixed_ms, fp64_ms, ir_ms], [], world, "cuda")

    # end to end through the public C-ABI with pinned host buffers
    rhs_pin = torch.from_numpy(rhs_h).pin_memory()
    x_pin = torch.zeros(n, dtype=torch.float64).pin_memory()
    e2e_ms = []
    for k in range(args.steps + 1):
        x_pin.zero_()
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = _lib.StatsC()
        solver.ctx.call("tpa_solve", _lib.ptr(rhs_pin.numpy(), C.c_double), _lib.ptr(x_pin.numpy(), C.c_double),
                        RTOL, 0.0, 100, 0, 1, C.byref(st))
        dt = (time.perf_counter() - t0) * 1e3
        if k:
            e2e_ms.append(dt)
        e2e_it = st.cycles
    e2e_ms_mean = float(np.mean(e2e_ms))

    # roofline of the dominant kernel, timed alone (CUDA events, 200 launches):
    # with the finest level on CSR tiles or row-streamed its down kernel (both
    # pre-sweeps, the residual and the restriction), else the smoothing sweep
    skappa = 0 if args.workload == "uniform_2048" else 1
    sweep, sweep64 = C.c_double(), C.c_double()

    def down_kernel(which, name):
        solver.ctx.call("tpa_time_kernel", which, 0, 1, 200, C.byref(sweep))
        solver.ctx.call("tpa_time_kernel", which, 0, 0, 200, C.byref(sweep64))
        # read the FP64 residual (and two face coefficients when they vary),
        # write the pre-smoothed iterate, the projected RHS and the coarse RHS
        # (a quarter of a value per fine cell): 8 + 2 s_kappa + 2 s + s / 4
        return name, n * (8 + 2 * 4 * skappa + 2 * 4 + 1)

    try:
        try:
            kname, alg32 = down_kernel(6, "k_tile_down, finest level, FP32 cycle (both pre-sweeps, residual, "
                                          "restriction)")
        except _lib.TpaError:
            kname, alg32 = down_kernel(8, "v_stream_down, finest level, FP32 cycle (row-streamed: both "
                                          "pre-sweeps, residual, restriction)")
    except _lib.TpaError:
        solver.ctx.call("tpa_time_kernel", 0, 0, 1, 200, C.byref(sweep))
        solver.ctx.call("tpa_time_kernel", 0, 0, 0, 200, C.byref(sweep64))
        # one damped-Jacobi sweep: read x and b, write x, plus two face
        # coefficients per cell when they vary (3 s + 2 s_kappa)
        kname = "damped-Jacobi sweep, finest level, FP32"
        alg32 = n * (3 * 4 + 2 * 4 * skappa)
    peak, peak_kind = measured_peaks()
    achieved = alg32 / (sweep.value * 1e-3) / 1e9

    # the same solve with the red-black Gauss-Seidel smoother (an option; the
    # reference smooths with damped Jacobi), after the timed solves
    red_black = None
    if not args.profile:
        from tpagmg import MultigridOptions
        rb = EllipticSolver(PoissonOperator(mesh, kappa), device=local,
                            multigrid=MultigridOptions(smoother="red_black"))
        rb.ctx.call("tpa_set_stream", C.c_void_p(stream.cuda_stream))

        def rb_timed(precision, steps):
            ms, its = [], []
            for k in range(steps + 2):
                x_d.zero_()
                flush.fill_(1.0)
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                st = rb.solve_device(rhs_d.data_ptr(), x_d.data_ptr(), rtol=RTOL, precision=precision)
                e1.record(stream)
                e1.synchronize()
                assert st.converged, st
                if k >= 2:
                    ms.append(e0.elapsed_time(e1))
                    its.append(st.cycles)
            return float(np.mean(ms)), float(np.mean(its))
        rb_mixed_ms, rb_mixed_it = rb_timed("mixed", args.steps)
        rb_fp64_ms, rb_fp64_it = rb_timed("fp64", args.steps)
        red_black = {"mixed_ms": rb_mixed_ms, "fp64_ms": rb_fp64_ms,
                     "cg_iterations": {"mixed": rb_mixed_it, "fp64": rb_fp64_it},
                     "mixed_value": world * n * rb_mixed_it / (rb_mixed_ms * 1e-3),
                     "what": "red-black Gauss-Seidel smoother (MultigridOptions smoother='red_black'), "
                             "same inputs and tolerance, default layout"}
        del rb

    # the per-step coefficient refresh (`_refresh_geometric_multigrid!`), after
    # the timed solves: device path, then the host path, median wall ms
    refresh = None
    if args.workload == "droplet_amr":
        def refresh_ms(reps, host):
            if host:
                os.environ["TPAGMG_HOST_REFRESH"] = "1"
            out, path = [], None
            try:
                for k in range(reps):
                    solver.refresh(kappa * (1.0 + 0.01 * (k % 3)))
                    path, ms = solver.last_refresh()
                    out.append(ms)
            finally:
                os.environ.pop("TPAGMG_HOST_REFRESH", None)
            return path, float(np.median(out))
        solver.refresh(kappa)  # the first device refresh lists the entry terms (set-up)
        dpath, dms = refresh_ms(10, False)
        hpath, hms = refresh_ms(3, True)
        solver.refresh(kappa)
        refresh = {"device_ms": dms, "device_path": dpath, "host_ms": hms, "host_path": hpath,
                   "what": "tpa_refresh wall time: new face coefficients -> every level operator, "
                           "Jacobi and transfer weights, coarse inverse"}

    # one device-resident two-phase pressure step (two_phase/stepping.jl:73-111):
    # fractions -> conditional fractions -> kappa -> hierarchy refresh -> CGFM
    # force -> u* = u + dt a -> project! (mixed solve, default tolerance)
    two_phase = None
    if args.workload == "droplet_amr":
        from tpagmg import projection as P
        step = P.TwoPhaseStep(solver, (1000.0, 1.0), sigma=0.072, curvature=1.0 / 0.15)
        frac_d = torch.from_numpy(frac).cuda()
        u_d = torch.zeros(mesh.nfaces, dtype=torch.float64, device="cuda")
        ub_d = torch.zeros(max(mesh.nboundary_faces, 1), dtype=torch.float64, device="cuda")
        p_d = torch.zeros(n, dtype=torch.float64, device="cuda")
        dt = 1e-3

        def tp_step():
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record(stream)
            step.update_interface(frac_d)
            u_d.add_(step.force(), alpha=dt)
            st = step.project(u_d, ub_d, p_d, dt, precision="mixed")
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3, st

        for _ in range(3):
            tp_step()
        runs = [tp_step() for _ in range(10)]
        last, tp_path = runs[-1][2], solver.last_refresh()[0]
        os.environ["TPAGMG_HOST_REFRESH"] = "1"
        try:
            host_runs = [tp_step() for _ in range(3)]
        finally:
            os.environ.pop("TPAGMG_HOST_REFRESH", None)
        two_phase = {"device_ms": float(np.median([r[0] for r in runs])),
                     "wall_ms": float(np.median([r[1] for r in runs])),
                     "wall_ms_host_refresh": float(np.median([r[1] for r in host_runs])),
                     "refresh_path": tp_path,
                     "cg_iterations": last.cycles, "converged": last.converged,
                     "max_velocity_after": float(u_d.abs().max()),
                     "what": "fractions -> kappa -> refresh -> CGFM force -> u += dt a -> project! "
                             "(all fields on the device; dt 1e-3, tolerance sqrt(eps))"}
        solver.refresh(kappa)

    # the CMDGFM two-block solve on the capillary wave (not timed with the solves above)
    cmdgfm = None
    if args.workload == "droplet_amr" and rank == 0:
        cmdgfm = cmdgfm_measure(args.cmdgfm_level, args.steps, args.warmup, cpu=world == 1 and not args.no_cpu_baseline)

    cpu, oracle_err = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload == "droplet_amr":
        # the C/OpenMP restatement on this host's cores: the same measurement as
        # `--impl reference` (median of warm solves), then the FP64 oracle
        # solution of the very RHS the GPU solved, to rtol 1e-12, against which
        # both GPU solutions (rtol 1e-10) are compared
        from oracle import cgmg
        problem = cgmg.droplet_problem(args.levels)
        res = cgmg.bench_droplet(steps=10, warmup=3, threads=os.cpu_count(), problem=problem)
        cpu = {"value": res["cell_updates_per_s"], "unit": "cell-updates/s", "cores": res["threads"],
               "kind": "port", "sample": f"median of 10 warm full solves of the same droplet workload "
                                         f"(3 untimed), {res['threads']} OpenMP threads, setup excluded"}
        x_oracle, ost = res["runner"].solve(rhs_h, rtol=1e-12, threads=os.cpu_count())
        ref_max = float(np.max(np.abs(x_oracle)))
        oracle_err = {"mixed": float(np.max(np.abs(x_mixed.cpu().numpy() - x_oracle)) / ref_max),
                      "fp64": float(np.max(np.abs(x_ref.cpu().numpy() - x_oracle)) / ref_max),
                      "mixed_ir": float(np.max(np.abs(x_ir.cpu().numpy() - x_oracle)) / ref_max),
                      "norm": "max |x_gpu - x_oracle| / max |x_oracle|",
                      "oracle": f"C restatement solved to rtol 1e-12 ({ost.cycles} CG iterations) on the same RHS"}
    # DRAM bytes per launch of the roofline kernel from a committed ncu capture
    traffic = None
    tp = ROOT / "profiles" / "roofline_traffic.json"
    if tp.exists():
        rec = json.loads(tp.read_text()).get(args.workload)
        if rec:
            traffic = rec["dram_bytes_per_launch"]

    cells_updates = n * mixed_it
    value = world * cells_updates / (mixed_ms * 1e-3)
    if args.workload == "droplet_amr":
        metric = DROPLET_METRIC
        wname = f"droplet_amr levels={args.levels} (unit square, 4x4 roots of 16x16, circle band)"
    else:
        metric = f"cell-updates/s to rel. residual 1e-10 ({args.size}^2 uniform periodic solve, mixed FP32/FP64 GMG)"
        wname = f"uniform_{args.size} (periodic unit square, {args.size // 16}x{args.size // 16} roots of 16x16)"
    line = {
        "metric": metric,
        "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": mixed_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32/f64", "data": "synthetic (seeded Philox)",
        "config": {"workload": wname,
                   "fine_cells": n, "levels": solver.level_sizes(), "parallelism": "replicas" if world > 1 else "1 GPU",
                   "l2": "flushed between steps (256 MiB write)", "device_layout": dict(solver.device_info(), tiled_levels=solver.tiled_levels()),
                   "autotuned_layout": layout, "autotuned_layout_fp64": layouts.get("fp64"), "autotune_s": tune_s},
        "time_to_tolerance_ms": {"mixed": mixed_ms, "fp64": fp64_ms, "speedup_mixed_over_fp64": fp64_ms / mixed_ms,
                                 "mixed_ir": ir_ms, "speedup_mixed_ir_over_fp64": fp64_ms / ir_ms},
        "cg_iterations": {"mixed": mixed_it, "fp64": fp64_it, "mixed_ir": ir_it},
        "precisions": {"mixed": "FP32 V-cycle, FP64 Krylov vectors",
                       "fp64": "FP64 V-cycle and Krylov vectors",
                       "mixed_ir": "FP32 V-cycle and Krylov vectors (r, p, Ap, z) inside FP64 iterative refinement: "
                                   "FP64 iterate, true residual and inner products"},
        "mixed_ir_error_vs_fp64": ir_err,
        "fp64_value": world * n * fp64_it / (fp64_ms * 1e-3),
        "mixed_error_vs_fp64": mixed_err,
        "error_vs_fp64_oracle": oracle_err,
        "e2e": {"value": world * n * e2e_it / (e2e_ms_mean * 1e-3), "unit": "cell-updates/s",
                "ms_per_step": e2e_ms_mean, "h2d_bytes_per_step": 2 * 8 * n, "d2h_bytes_per_step": 8 * n},
        "gpu_launches": mixed_launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": kname,
                     "kernel_ms": sweep.value, "kernel_ms_fp64": sweep64.value,
                     "algorithmic_bytes": alg32, "peak_kind": peak_kind},
        "whole_solve_roofline": whole_solve_roofline(n, skappa, (mixed_it, mixed_ms), (fp64_it, fp64_ms), peak,
                                                     peak_kind, world),
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
        "refresh": refresh,
        "two_phase_step": two_phase,
        "red_black_smoother": red_black,
        "cmdgfm": cmdgfm,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
