"""The B200 solve against the oracle at the sizes of the benchmark workloads,
and against the reference's own generated solver checks.

* The reference's Chapter 11 solver checks (docs/techref/figures/generated/
  checks.tex, written by docs/techref/figures/solvers.jl from its own solves):
  the FP64 GPU solve takes exactly the reference's PCG iteration count on
  every case, with its level count and convergence factor; the mixed solve
  converges in at most one more iteration.
* The two-phase droplet at its benchmark depth (4 levels, 110,080 cells,
  density ratio 1000): GPU FP64 (rtol 1e-12) against the C restatement of the
  oracle solve (rtol 1e-12) to 1e-10; the GPU solves at the benchmark's rtol
  1e-10 to 1e-9 (FP64 and mixed).
* The uniform periodic 2048^2 solve (4.19M cells): against the exact solution
  of the same discrete system (FFT), to 1e-10 (FP64, rtol 1e-12) and 1e-9
  (mixed and FP64 at rtol 1e-10).
* Merged batches with problems of tree depth 5 and 6: every problem against
  its own oracle solve, 1e-10 (FP64) and 1e-9 (mixed).

Errors are max |x - x_oracle| / max |x_oracle|; both sides remove the volume
mean, so the gauge is the same.
"""
import numpy as np
import pytest

from oracle import cgmg
from oracle import fft_poisson as F
from oracle import projection as OP
from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions as OMG, TreeGeometricMultigrid
from oracle.operator import PoissonOperator as OOp

pytestmark = pytest.mark.gpu

from tpagmg import BatchedSolver, BlockTreeMesh, EllipticSolver, PoissonOperator, solve  # noqa: E402
from tpagmg import workloads as W  # noqa: E402
import reference_cases as RC  # noqa: E402

GOLD = __import__("json").loads((__import__("pathlib").Path(__file__).parent / "golden" /
                                 "known_answers.json").read_text())["techref_pressure_solves"]


def rel_err(x, ref):
    return float(np.max(np.abs(x - ref)) / np.max(np.abs(ref)))


def oracle_solution(spec, kappa, rhs, rtol=1e-12):
    """The FP64 oracle solve: the Python oracle's hierarchy, solved by its C
    restatement (tests/test_oracle_cgmg.py pins the two together)."""
    op = OOp(block_tree_mesh(**spec), kappa)
    mg = TreeGeometricMultigrid(op, OMG())
    x, st = cgmg.Runner(op, mg).solve(rhs, rtol=rtol)
    assert st.converged
    return x


@pytest.mark.parametrize("name", list(RC.TECHREF_CASES))
def test_gpu_takes_the_reference_iteration_counts(name):
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
    assert m.ncells == ref["unknowns"] and len(s.level_sizes()) == ref["levels"]
    x = np.zeros(m.ncells)
    st = solve(x, s, rhs, rtol=1e-10, max_cycles=20000, precision="fp64")
    assert st.converged and st.cycles == ref["cycles"]
    assert f"{(st.final_l2 / st.initial_l2) ** (1.0 / st.cycles):.2f}" == ref["factor"]
    xm = np.zeros(m.ncells)
    stm = solve(xm, s, rhs, rtol=1e-10, max_cycles=20000, precision="mixed")
    assert stm.converged and ref["cycles"] <= stm.cycles <= ref["cycles"] + 1


def test_droplet_benchmark_size_matches_oracle():
    spec = W.droplet_spec(levels=4)
    m = BlockTreeMesh(**spec)
    assert m.ncells == 110080
    _, kappa, psi = W.droplet_inputs(m)
    s = EllipticSolver(PoissonOperator(m, kappa))
    rhs = W.droplet_rhs(m, s.apply(psi))
    xo = oracle_solution(spec, kappa, rhs)
    errs = {}
    for precision, rtol, tol in (("fp64", 1e-12, 1e-10), ("fp64", 1e-10, 1e-9), ("mixed", 1e-10, 1e-9)):
        x = np.zeros(m.ncells)
        st = solve(x, s, rhs, rtol=rtol, precision=precision)
        assert st.converged
        errs[(precision, rtol)] = rel_err(x, xo)
        assert errs[(precision, rtol)] <= tol, (precision, rtol, errs)
    print("droplet levels=4 error vs FP64 oracle:", errs)


def test_uniform_2048_matches_exact_solution():
    spec = W.uniform_spec(2048)
    m = BlockTreeMesh(**spec)
    assert m.ncells == 2048 * 2048
    s = EllipticSolver(PoissonOperator(m, np.ones(m.nfaces)))
    rhs = W.gaussian_rhs(m, W.SEEDS["uniform_2048"])
    xo = F.solve(rhs, spec["base_mesh"], spec["block_size"], spec.get("extent", (1.0, 1.0)))
    errs = {}
    for precision, rtol, tol in (("fp64", 1e-12, 1e-10), ("fp64", 1e-10, 1e-9), ("mixed", 1e-10, 1e-9)):
        x = np.zeros(m.ncells)
        st = solve(x, s, rhs, rtol=rtol, precision=precision)
        assert st.converged
        errs[(precision, rtol)] = rel_err(x, xo)
        assert errs[(precision, rtol)] <= tol, (precision, rtol, errs)
    print("uniform 2048^2 error vs exact solution:", errs)


def test_merged_batch_deep_problems_match_oracle():
    problems = W.batch_problems(256)
    pick = [next(p for p in problems if p["depth"] == d) for d in (6, 5, 2, 3)]
    built = []
    for p in pick:
        spec = W.batch_spec(p)
        m = BlockTreeMesh(**spec)
        kappa, rhs = W.batch_inputs(m, p)
        built.append((spec, m, kappa, rhs, EllipticSolver(PoissonOperator(m, kappa))))
    batch = BatchedSolver([b[4] for b in built])
    rhs_all = batch.concat([b[3] for b in built])
    oracles = [oracle_solution(spec, kappa, rhs) for spec, _, kappa, rhs, _ in built]
    for precision, tol in (("fp64", 1e-10), ("mixed", 1e-9)):
        x = np.zeros(batch.ncells)
        stats = batch.solve(x, rhs_all, rtol=1e-12 if precision == "fp64" else 1e-10, precision=precision)
        assert all(st["converged"] for st in stats)
        for k, (xk, xo) in enumerate(zip(batch.split(x), oracles)):
            assert rel_err(xk, xo) <= tol, (precision, pick[k]["depth"], rel_err(xk, xo))
