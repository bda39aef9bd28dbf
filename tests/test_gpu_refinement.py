"""The refinement solve (precision "mixed_ir", tpa_solve precision 2): FP64
iterative refinement around CG runs whose r, p, Ap and z are stored in FP32,
the V-cycle in FP32, and the iterate, the true residual that starts each run
and every inner product in FP64.  It has no counterpart in the reference; its
answers are held to those of the FP64 path:

* the two benchmark workloads at full size: the droplet (4 levels, 110,080
  cells) against the C restatement of the oracle solve, the uniform 2048^2
  against the exact solution of the discrete system (FFT), both to 1e-9 at
  rtol 1e-10, with the final FP64 true residual at or below the target and at
  most three more CG iterations than the FP64 solve;
* the reference's generated solver checks (uniform, AMR and drop cases):
  converged, within three iterations of the reference's PCG count, and equal
  to the FP64 solve to 1e-9;
* a nonzero initial guess, a zero right-hand side, an operator with open
  sides (no nullspace) and the projection step;
* the merged batch rejects it.

Errors are max |x - x_ref| / max |x_ref|; every solution has its volume mean
removed, so the gauge is the same."""
import numpy as np
import pytest

from oracle import fft_poisson as F
from oracle import projection as OP

pytestmark = pytest.mark.gpu

from tpagmg import BatchedSolver, BlockTreeMesh, EllipticSolver, MultigridOptions, PoissonOperator, solve  # noqa: E402
from tpagmg import projection as P  # noqa: E402
from tpagmg import workloads as W  # noqa: E402
from tpagmg._lib import TpaError  # noqa: E402
import reference_cases as RC  # noqa: E402
from test_gpu_fullsize import GOLD, oracle_solution, rel_err  # noqa: E402


def check_refined(s, rhs, xref, tol=1e-9, rtol=1e-10):
    x64 = np.zeros(s.operator.mesh.ncells)
    st64 = solve(x64, s, rhs, rtol=rtol, precision="fp64")
    x = np.zeros(s.operator.mesh.ncells)
    st = solve(x, s, rhs, rtol=rtol, precision="mixed_ir")
    assert st.converged and st.final_linf <= st.target_linf
    assert st.cycles <= st64.cycles + 3, (st.cycles, st64.cycles)
    err = rel_err(x, xref)
    assert err <= tol, err
    return st, st64, err


def test_droplet_benchmark_size():
    spec = W.droplet_spec(levels=4)
    m = BlockTreeMesh(**spec)
    _, kappa, psi = W.droplet_inputs(m)
    s = EllipticSolver(PoissonOperator(m, kappa))
    rhs = W.droplet_rhs(m, s.apply(psi))
    st, st64, err = check_refined(s, rhs, oracle_solution(spec, kappa, rhs))
    print("droplet levels=4, mixed_ir:", st.cycles, "CG iterations in", st.restarts, "runs (FP64:",
          st64.cycles, "); error vs FP64 oracle", err)


def test_uniform_2048():
    spec = W.uniform_spec(2048)
    m = BlockTreeMesh(**spec)
    s = EllipticSolver(PoissonOperator(m, np.ones(m.nfaces)))
    rhs = W.gaussian_rhs(m, W.SEEDS["uniform_2048"])
    xo = F.solve(rhs, spec["base_mesh"], spec["block_size"], spec.get("extent", (1.0, 1.0)))
    st, st64, err = check_refined(s, rhs, xo)
    print("uniform 2048^2, mixed_ir:", st.cycles, "CG iterations in", st.restarts, "runs (FP64:", st64.cycles,
          "); error vs exact", err)


@pytest.mark.parametrize("name", list(RC.TECHREF_CASES))
def test_reference_solver_checks(name):
    maker, n, drop = RC.TECHREF_CASES[name]
    ref = GOLD["solves"][name]
    m = BlockTreeMesh(**maker(n))
    kappa = np.ones(m.nfaces)
    if drop:
        frac = W.circle_fractions(m, RC.TECHREF_CENTRE, RC.TECHREF_RADIUS)
        _, cond = OP.conditional_fraction(frac)
        kappa = OP.face_coefficients(m, cond, RC.TECHREF_DENSITY)
    s = EllipticSolver(PoissonOperator(m, kappa))
    rhs = RC.techref_noise(m.ncells)
    xr = np.zeros(m.ncells)
    assert solve(xr, s, rhs, rtol=1e-12, precision="fp64").converged
    x = np.zeros(m.ncells)
    st = solve(x, s, rhs, rtol=1e-10, max_cycles=20000, precision="mixed_ir")
    assert st.converged and st.cycles <= ref["cycles"] + 3, (st.cycles, ref["cycles"])
    assert rel_err(x, xr) <= 1e-9


def test_initial_guess_zero_rhs_and_open_sides():
    spec = dict(base_mesh=(64, 64), block_size=(16, 16), periodic=(False, False))
    m = BlockTreeMesh(**spec)
    s = EllipticSolver(PoissonOperator(m))
    rng = np.random.default_rng(21)
    rhs = rng.standard_normal(m.ncells)
    rhs -= np.sum(rhs * m.cell_volumes()) / np.sum(m.cell_volumes())
    xr = np.zeros(m.ncells)
    assert solve(xr, s, rhs, rtol=1e-12, precision="fp64").converged
    # a warm start (its mean is removed first).  Its residual is far above the
    # right-hand side, so the target is absolute: that of a cold start at rtol
    # 1e-10 (the strong residual of x = 0 is max |rhs|)
    x = rng.standard_normal(m.ncells)
    st = solve(x, s, rhs, rtol=0.0, atol=1e-10 * np.max(np.abs(rhs)), precision="mixed_ir")
    assert st.converged and st.restarts >= 2
    assert rel_err(x, xr) <= 1e-9
    z = np.zeros(m.ncells)
    st = solve(z, s, np.zeros(m.ncells), precision="mixed_ir")
    assert st.converged and st.cycles == 0 and np.all(z == 0)
    # open left and right sides: every level non-singular, a nonzero-mean RHS
    so = EllipticSolver(PoissonOperator(m, 1.0, velocity_boundary=(True, True, False, False)),
                        multigrid=MultigridOptions())
    rhs1 = np.cos(np.arange(m.ncells))
    xo = np.zeros(m.ncells)
    assert solve(xo, so, rhs1, rtol=1e-12, compatibility="error", precision="fp64").converged
    xi = np.zeros(m.ncells)
    st = solve(xi, so, rhs1, rtol=1e-10, compatibility="error", precision="mixed_ir")
    assert st.converged and st.removed_rhs_mean == 0.0
    assert rel_err(xi, xo) <= 1e-9


def test_projection_step():
    """project! with the refinement solve: the same velocity and pressure as
    with the FP64 solve, to 1e-9 of their scale."""
    import torch
    spec = W.droplet_spec(levels=2)
    m = BlockTreeMesh(**spec)
    _, kappa, _ = W.droplet_inputs(m)
    s = EllipticSolver(PoissonOperator(m, kappa))
    rng = np.random.default_rng(5)
    u = rng.standard_normal(m.nfaces)
    out = {}
    for precision in ("fp64", "mixed_ir"):
        ud = torch.from_numpy(u.copy()).cuda()
        ubd = torch.zeros(m.nboundary_faces, dtype=torch.float64, device="cuda")
        pd = torch.zeros(m.ncells, dtype=torch.float64, device="cuda")
        st = P.project_device(ud, ubd, pd, s, 1e-3, tolerance=1e-12, precision=precision)
        assert st.converged
        out[precision] = (ud.cpu().numpy(), pd.cpu().numpy())
    (u64, p64), (uir, pir) = out["fp64"], out["mixed_ir"]
    assert np.max(np.abs(uir - u64)) <= 1e-9 * np.max(np.abs(u64))
    assert rel_err(pir, p64) <= 1e-9


def test_batch_rejects_refinement():
    m = BlockTreeMesh(base_mesh=(32, 32), block_size=(16, 16), periodic=(True, True))
    batch = BatchedSolver([EllipticSolver(PoissonOperator(m))])
    with pytest.raises(TpaError):
        batch.solve(np.zeros(batch.ncells), np.zeros(batch.ncells), precision="mixed_ir")
