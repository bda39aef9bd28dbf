"""The CMDGFM solve's oracle and the library's host set-up, on the CPU.

* The library's Schur complement and incomplete LU (tpa_cmdgfm_factor, host
  code) equal the oracle's restatement bit for bit: both sum in the orders
  oracle/cmdgfm.py documents.
* The Schur complement is J - C D^-1 B to 1e-13 (the reference's own check,
  test/two_phase/two_velocity/projection/cmdgfm_projection.jl:331-342).
* Without dropping, the Crout ILU is the exact LU without pivoting.
* BiCGSTAB (Krylov.jl 0.10 restated) solves a nonsymmetric system, and the
  residual-replacement loop with the block preconditioner recovers the exact
  solution of the synthetic capillary-wave system below the reference's
  default tolerance sqrt(eps).
* An empty jump block, and the C-ABI's argument checks.

The synthetic system (tpagmg.workloads.cmdgfm_system) has the reference's
block structure on the mesh of examples/07_capillary_wave; the reference's
own CMDGFM tests assemble it from its interface geometry, which this
library leaves to the caller."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import cmdgfm as O
from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions, TreeGeometricMultigrid
from oracle.operator import PoissonOperator as OOp

from tpagmg import BlockTreeMesh, EllipticSolver, PoissonOperator  # noqa: E402
from tpagmg import workloads as W  # noqa: E402
from tpagmg._lib import TpaError  # noqa: E402
from tpagmg.cmdgfm import CMDGFMSystem, cmdgfm_factor  # noqa: E402
from tpagmg.operator import mixture_density  # noqa: E402


def wave_case(level):
    spec = W.capillary_wave_spec(level)
    m = BlockTreeMesh(**spec)
    fr = W.wave_fractions(m)
    kappa = 1.0 / mixture_density(m, fr, (1.0, 1e-3))
    s = EllipticSolver(PoissonOperator(m, kappa))
    system, exact = W.cmdgfm_system(m, s.level_matrix(0), kappa, fr)
    return spec, m, kappa, system, exact


def oracle_system(system):
    M = sp.csr_matrix((system.val, system.col, system.row_ptr), shape=(system.n, system.n))
    E = sp.csr_matrix((system.extra_val, system.extra_col, system.extra_row_ptr),
                      shape=(len(system.extra_row_ptr) - 1, system.n))
    return O.CMDGFMSystem(matrix=M, rhs=system.rhs, np_=system.np_, pressure_cell=system.pressure_cell,
                          pressure_anchor=system.pressure_anchor, defect_weight=system.defect_weight, extra=E,
                          extra_rhs=system.extra_rhs, extra_weight=system.extra_weight,
                          row_scale=system.row_scale, col_scale=system.col_scale,
                          drop_tolerance=system.drop_tolerance, tolerance=system.tolerance,
                          max_iterations=system.max_iterations, warm_start=system.warm_start,
                          initial_pressure=system.initial_pressure)


def rows_to_csr(rows, n):
    ptr, col, val = [0], [], []
    for r in rows:
        for c, v in r.items():
            col.append(c)
            val.append(v)
        ptr.append(len(col))
    return np.array(ptr), np.array(col, dtype=np.int64), np.array(val)


@pytest.mark.parametrize("level", [2, 4])
def test_library_factor_equals_oracle_bitwise(level):
    _, _, _, system, _ = wave_case(level)
    (s_ptr, s_col, s_val), (l_ptr, l_col, l_val), (u_ptr, u_col, u_val) = cmdgfm_factor(system)
    M = sp.csr_matrix((system.val, system.col, system.row_ptr), shape=(system.n, system.n))
    S = O.schur_complement(M, system.np_)
    L, U = O.ilu_crout(S, system.drop_tolerance)
    for (ptr, col, val), rows in (((s_ptr, s_col, s_val), S), ((l_ptr, l_col, l_val), L)):
        optr, ocol, oval = rows_to_csr(rows, system.nx)
        assert np.array_equal(ptr, optr) and np.array_equal(col, ocol)
        assert np.array_equal(val, oval)  # bit for bit
    # U: the pivot first in each row, then the rest in column order
    uptr, ucol, uval = [0], [], []
    for k, r in enumerate(U):
        ucol.append(k)
        uval.append(r[k])
        for c, v in r.items():
            if c != k:
                ucol.append(c)
                uval.append(v)
        uptr.append(len(ucol))
    assert np.array_equal(u_ptr, uptr) and np.array_equal(u_col, ucol) and np.array_equal(u_val, uval)


def test_schur_complement_is_j_minus_c_dinv_b():
    _, _, _, system, _ = wave_case(3)
    M = sp.csr_matrix((system.val, system.col, system.row_ptr), shape=(system.n, system.n)).toarray()
    npr = system.np_
    A, B, Cm, J = M[:npr, :npr], M[:npr, npr:], M[npr:, :npr], M[npr:, npr:]
    expected = J - Cm @ (B / np.diag(A)[:, None])
    sp_, scol, sval = cmdgfm_factor(system)[0]
    S = sp.csr_matrix((sval, scol, sp_), shape=(system.nx, system.nx)).toarray()
    assert np.allclose(S, expected, rtol=1e-13, atol=1e-13 * np.abs(expected).max())
    assert not np.array_equal(S, J)


def test_crout_ilu_without_dropping_is_exact_lu():
    rng = np.random.default_rng(3)
    n = 40
    Adense = rng.standard_normal((n, n)) * (rng.random((n, n)) < 0.15) + np.diag(6 + rng.random(n))
    rows = [{j: Adense[i, j] for j in range(n) if Adense[i, j] != 0} for i in range(n)]
    L, U = O.ilu_crout(rows, 0.0)
    Ld = np.eye(n)
    Ud = np.zeros((n, n))
    for k in range(n):
        for c, v in L[k].items():
            Ld[k, c] = v
        for c, v in U[k].items():
            Ud[k, c] = v
    assert np.allclose(Ld @ Ud, Adense, atol=1e-12)
    b = rng.standard_normal(n)
    assert np.allclose(O.ilu_solve(L, U, b), np.linalg.solve(Adense, b), atol=1e-10)


def test_bicgstab_solves_a_nonsymmetric_system():
    rng = np.random.default_rng(9)
    n = 60
    A = np.diag(4 + rng.random(n)) + 0.5 * rng.standard_normal((n, n)) * (rng.random((n, n)) < 0.1)
    b = rng.standard_normal(n)
    x, its, status = O.bicgstab(lambda v: A @ v, None, b, 0.0, 1e-12, 200)
    assert status == "solution good enough" and 0 < its < 60
    assert np.allclose(x, np.linalg.solve(A, b), rtol=1e-9, atol=1e-9)
    # right preconditioning by the exact inverse: one iteration
    Ainv = np.linalg.inv(A)
    x, its, _ = O.bicgstab(lambda v: A @ v, lambda v: Ainv @ v, b, 0.0, 1e-10, 200)
    assert its == 1 and np.allclose(x, np.linalg.solve(A, b), rtol=1e-9)


def test_oracle_solve_recovers_the_exact_solution():
    spec, m, kappa, system, exact = wave_case(3)
    om = block_tree_mesh(**spec)
    oop = OOp(om, kappa)
    M = sp.csr_matrix((system.val, system.col, system.row_ptr), shape=(system.n, system.n))
    # the pressure block is the oracle operator's matrix (anchor removed)
    assert abs(M[:system.np_, :system.np_] - oop.matrix[1:, 1:]).max() <= 1e-12 * abs(oop.matrix).max()
    mg = TreeGeometricMultigrid(oop, MultigridOptions())
    x, st = O.solve(oracle_system(system), mg)
    assert st.converged and st.iterations < 100, st
    assert max(st.pressure_defect, st.jump_defect, st.anchor_defect) <= system.tolerance
    npr = system.np_
    assert np.max(np.abs(x[:npr] - exact[:npr])) <= 1e-6 * np.max(np.abs(exact[:npr]))
    assert np.max(np.abs(x[npr:] - exact[npr:])) <= 1e-6 * np.max(np.abs(exact[npr:]))
    # without the preconditioner BiCGSTAB needs far more iterations
    x0, st0 = O.solve(oracle_system(system), mg, preconditioned=False)
    assert st0.iterations > 3 * st.iterations


def test_empty_jump_block_and_argument_checks():
    spec, m, kappa, system, _ = wave_case(2)
    # the pressure block alone (no mixed face)
    npr = system.np_
    M = sp.csr_matrix((system.val, system.col, system.row_ptr), shape=(system.n, system.n))[:npr, :npr].tocsr()
    M.sort_indices()
    E = sp.csr_matrix((system.extra_val, system.extra_col, system.extra_row_ptr),
                      shape=(1, system.n))[:, :npr].tocsr()
    pure = CMDGFMSystem(np_=npr, row_ptr=M.indptr, col=M.indices, val=M.data, rhs=system.rhs[:npr],
                        pressure_cell=system.pressure_cell, pressure_anchor=system.pressure_anchor,
                        defect_weight=system.defect_weight[:npr], extra_row_ptr=E.indptr, extra_col=E.indices,
                        extra_val=E.data, extra_rhs=system.extra_rhs, extra_weight=system.extra_weight,
                        row_scale=system.row_scale[:npr], col_scale=system.col_scale[:npr])
    s_, l_, u_ = cmdgfm_factor(pure)
    assert len(s_[1]) == len(l_[1]) == len(u_[1]) == 0
    bad = []
    for field, value in (("col_scale", -system.col_scale), ("tolerance", 0.0), ("max_iterations", 0),
                         ("drop_tolerance", -1.0)):
        kw = dict(system.__dict__)
        kw[field] = value
        bad.append(CMDGFMSystem(**kw))
    unsorted = dict(system.__dict__)
    col = system.col.copy()
    r0, r1 = system.row_ptr[0], system.row_ptr[1]
    col[r0:r1] = col[r0:r1][::-1]
    unsorted["col"] = col
    bad.append(CMDGFMSystem(**unsorted))
    cells = dict(system.__dict__)
    cells["pressure_anchor"] = system.pressure_cell.copy()  # a cell anchoring itself
    bad.append(CMDGFMSystem(**cells))
    for b in bad:
        with pytest.raises(TpaError):
            cmdgfm_factor(b)


def test_warm_start_takes_a_good_guess_and_refuses_a_bad_one():
    """`_cmdgfm_initial_solution!` restated (cmdgfm_projection.jl:1973-2040):
    a previous increment near the solution is taken and saves iterations; one
    far from it is refused, and the solve ends at the same solution."""
    spec, m, kappa, system, exact = wave_case(3)
    oop = OOp(block_tree_mesh(**spec), kappa)
    mg = TreeGeometricMultigrid(oop, MultigridOptions())
    npr = system.np_
    _, cold = O.solve(oracle_system(system), mg)
    kw = dict(system.__dict__)
    rng = np.random.default_rng(4)
    kw.update(warm_start=True, initial_pressure=exact[:npr] * (1 + 1e-4 * rng.standard_normal(npr)))
    good = CMDGFMSystem(**kw)
    x, warm = O.solve(oracle_system(good), mg)
    assert warm.initial_guess_used and warm.converged and warm.iterations < cold.iterations
    assert np.max(np.abs(x[:npr] - exact[:npr])) <= 1e-6 * np.max(np.abs(exact[:npr]))
    kw.update(initial_pressure=exact[:npr] * 50.0)
    x, bad = O.solve(oracle_system(CMDGFMSystem(**kw)), mg)
    assert bad.converged
    assert np.max(np.abs(x[:npr] - exact[:npr])) <= 1e-6 * np.max(np.abs(exact[:npr]))
