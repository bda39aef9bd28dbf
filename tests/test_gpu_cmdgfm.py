"""The CMDGFM two-block solve on the B200 (tpa_cmdgfm_solve) against the
oracle's restatement (oracle/cmdgfm.py) on the synthetic capillary-wave
systems (tpagmg.workloads.cmdgfm_system, the mesh of examples/07_capillary_
wave at its own refinement, 4 levels, and at 6 levels):

* converged: every defect at or below the reference's default tolerance
  sqrt(eps), within two BiCGSTAB iterations of the oracle's count;
* the exact solution recovered to 1e-6 of its scale (the oracle's own bound in
  tests/test_oracle_cmdgfm.py), and the oracle's solution to the same;
* FP64 and FP32 V-cycles in the pressure block;
* a repeated solve gives the same bits (fixed-order reductions);
* an empty jump block, and cells outside the mesh rejected."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import cmdgfm as O
from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions, TreeGeometricMultigrid
from oracle.operator import PoissonOperator as OOp

pytestmark = pytest.mark.gpu

from tpagmg import BlockTreeMesh, EllipticSolver, PoissonOperator  # noqa: E402
from tpagmg import workloads as W  # noqa: E402
from tpagmg._lib import TPA_ERR_INVALID_ARG, TpaError  # noqa: E402
from tpagmg.cmdgfm import CMDGFMSystem, solve_cmdgfm  # noqa: E402
from tpagmg.operator import mixture_density  # noqa: E402
from test_oracle_cmdgfm import oracle_system  # noqa: E402

CASES = {}


def case(level):
    if level not in CASES:
        spec = W.capillary_wave_spec(level)
        m = BlockTreeMesh(**spec)
        fr = W.wave_fractions(m)
        kappa = 1.0 / mixture_density(m, fr, (1.0, 1e-3))
        s = EllipticSolver(PoissonOperator(m, kappa))
        system, exact = W.cmdgfm_system(m, s.level_matrix(0), kappa, fr)
        oop = OOp(block_tree_mesh(**spec), kappa)
        mg = TreeGeometricMultigrid(oop, MultigridOptions())
        xo, so = O.solve(oracle_system(system), mg)
        assert so.converged
        CASES[level] = (s, system, exact, xo, so)
        ORACLE_MG[level] = mg
    return CASES[level]


ORACLE_MG = {}


def rel(a, b, sl):
    return float(np.max(np.abs(a[sl] - b[sl])) / np.max(np.abs(b[sl])))


@pytest.mark.parametrize("level", [4, 6])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cmdgfm_matches_oracle(level, precision):
    s, system, exact, xo, so = case(level)
    x, st = solve_cmdgfm(s, system, precision=precision)
    assert st.converged, st
    assert max(st.pressure_defect, st.jump_defect, st.anchor_defect) <= system.tolerance
    assert abs(st.iterations - so.iterations) <= 2, (st.iterations, so.iterations)
    npr = system.np_
    for part in (slice(0, npr), slice(npr, system.n)):
        assert rel(x, exact, part) <= 1e-6
        assert rel(x, xo, part) <= 1e-6
    assert st.lower_levels >= 1 and st.upper_levels >= 1 and st.factor_entries > 0
    print(f"capillary wave L{level} ({precision}): n = {system.n}, nx = {system.nx}, {st.iterations} iterations "
          f"(oracle {so.iterations}), {st.device_ms:.2f} ms on the device, set-up {st.setup_ms:.2f} ms, "
          f"factor levels {st.lower_levels}/{st.upper_levels}")


def test_jump_block_paths_agree(monkeypatch):
    """The jump block through the factors' inverses (the default here) and
    by the row walk of the factors give the same iterates to rounding."""
    s, system, exact, xo, so = case(4)
    x_inv, st_inv = solve_cmdgfm(s, system)
    monkeypatch.setenv("TPAGMG_CMDGFM_WALK", "1")
    x_walk, st_walk = solve_cmdgfm(s, system)
    assert st_inv.inverse_entries > 0 and st_walk.inverse_entries == 0
    assert st_inv.iterations == st_walk.iterations
    assert np.max(np.abs(x_inv - x_walk)) <= 1e-9 * np.max(np.abs(x_walk))


def test_cmdgfm_repeats_bit_for_bit(monkeypatch):
    """A repeated solve, and the BiCGSTAB loop launched kernel by kernel
    instead of as one captured graph, give the same bits."""
    s, system, _, _, _ = case(4)
    x1, st1 = solve_cmdgfm(s, system)
    x2, st2 = solve_cmdgfm(s, system)
    assert np.array_equal(x1, x2) and st1.iterations == st2.iterations
    monkeypatch.setenv("TPAGMG_NO_GRAPH", "1")
    x3, st3 = solve_cmdgfm(s, system)
    assert np.array_equal(x1, x3) and st1.iterations == st3.iterations


def test_cmdgfm_pressure_block_alone_and_bad_cells():
    s, system, _, _, _ = case(4)
    npr = system.np_
    M = sp.csr_matrix((system.val, system.col, system.row_ptr), shape=(system.n, system.n))[:npr, :npr].tocsr()
    M.sort_indices()
    E = sp.csr_matrix((system.extra_val, system.extra_col, system.extra_row_ptr),
                      shape=(1, system.n))[:, :npr].tocsr()
    rng = np.random.default_rng(2)
    p_exact = rng.standard_normal(npr) * 1e4
    pure = CMDGFMSystem(np_=npr, row_ptr=M.indptr, col=M.indices, val=M.data, rhs=M @ p_exact,
                        pressure_cell=system.pressure_cell, pressure_anchor=system.pressure_anchor,
                        defect_weight=system.defect_weight[:npr], extra_row_ptr=E.indptr, extra_col=E.indices,
                        extra_val=E.data, extra_rhs=E @ p_exact, extra_weight=system.extra_weight,
                        row_scale=system.row_scale[:npr], col_scale=system.col_scale[:npr])
    x, st = solve_cmdgfm(s, pure)
    assert st.converged and st.lower_levels == 0
    assert np.max(np.abs(x - p_exact)) <= 1e-6 * np.max(np.abs(p_exact))
    kw = dict(system.__dict__)
    cells = system.pressure_cell.copy()
    cells[0] = s.operator.mesh.ncells  # one past the last cell
    kw["pressure_cell"] = cells
    with pytest.raises(TpaError) as e:
        solve_cmdgfm(s, CMDGFMSystem(**kw))
    assert e.value.code == TPA_ERR_INVALID_ARG


def test_warm_start_matches_oracle():
    """The warm start (`_cmdgfm_initial_solution!`): the GPU takes the same
    decision as the oracle, saves the same iterations (within two) and ends at
    the same solution, for a guess near the solution and for none."""
    s, system, exact, xo, so = case(4)
    npr = system.np_
    rng = np.random.default_rng(4)
    for guess in (exact[:npr] * (1 + 1e-4 * rng.standard_normal(npr)), None):
        kw = dict(system.__dict__)
        kw.update(warm_start=True, initial_pressure=guess)
        warm = CMDGFMSystem(**kw)
        xw_o, so_w = O.solve(oracle_system(warm), ORACLE_MG[4])
        x, st = solve_cmdgfm(s, warm)
        assert st.converged and st.initial_guess_used == so_w.initial_guess_used
        assert abs(st.iterations - so_w.iterations) <= 2, (st.iterations, so_w.iterations)
        assert rel(x, exact, slice(0, npr)) <= 1e-6 and rel(x, xw_o, slice(0, npr)) <= 1e-6
        if guess is not None:
            assert st.initial_guess_used and st.iterations < so.iterations
