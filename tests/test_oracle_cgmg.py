"""The C/OpenMP restatement of the solve loop (`oracle/cgmg.c`) against the
Python oracle.  cgmg.c is the timed CPU baseline of bench.py (the reference
arm and the `cpu_baseline` leg) and the FP64 checker of the full-size GPU
tests, so it must give the Python oracle's solve: the same CG iteration count
and the same solution to 1e-10 (relative to max |x|), on the same hierarchy
and right-hand side, for every thread count."""
import numpy as np
import pytest

from oracle import cgmg
from oracle.krylov import solve
from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions, TreeGeometricMultigrid
from oracle.operator import PoissonOperator
from tpagmg import workloads as W
import reference_cases as RC
from test_oracle_golden import techref_operator


def _manufactured():
    mesh = block_tree_mesh(**RC.two_level_spec(8))
    op = PoissonOperator(mesh)
    x, y = mesh.cell_centers()
    return op, TreeGeometricMultigrid(op, MultigridOptions(coarse_size=8)), \
        8 * np.pi ** 2 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y)


def _techref(name):
    mesh, op = techref_operator(*RC.TECHREF_VCYCLE_CASES.get(name) or RC.TECHREF_CASES[name])
    return op, TreeGeometricMultigrid(op, MultigridOptions()), RC.techref_noise(mesh.ncells)


def _droplet():
    _, op, mg, rhs = cgmg.droplet_problem(levels=2)
    return op, mg, rhs


CASES = {"manufactured_b8": _manufactured, "drop32": lambda: _techref("drop32"),
         "amr32": lambda: _techref("amr32"), "droplet_levels2": _droplet}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("threads", [1, 4])
def test_cgmg_matches_python_oracle(name, threads):
    op, mg, rhs = CASES[name]()
    ref, st = solve(op, mg, rhs, rtol=1e-10)
    run = cgmg.Runner(op, mg)
    x, cst = run.solve(rhs, rtol=1e-10, threads=threads)
    assert st.converged and cst.converged
    assert cst.cycles == st.cycles
    assert np.max(np.abs(x - ref)) <= 1e-10 * np.max(np.abs(ref))
    assert cst.initial_linf == pytest.approx(st.initial_linf, rel=1e-12)
    assert cst.target == pytest.approx(st.target_linf, rel=1e-12)


def test_cgmg_tight_tolerance_and_warm_start():
    """rtol 1e-12 (the bench's oracle solution) and a nonzero initial guess
    (the warm start of `_run_krylov_reliably!`)."""
    op, mg, rhs = _techref("drop32")
    x0 = np.linspace(-1.0, 1.0, len(rhs))
    ref, st = solve(op, mg, rhs, x0, rtol=1e-12)
    x, cst = cgmg.Runner(op, mg).solve(rhs, x0, rtol=1e-12, threads=2)
    assert cst.cycles == st.cycles and cst.converged
    assert np.max(np.abs(x - ref)) <= 1e-11 * np.max(np.abs(ref))
