"""Pin the CPU oracle against the reference's own published known answers
(tests/golden/known_answers.json, extracted by make_known_answers.py)."""
import json
import pathlib

import numpy as np
import pytest

from oracle.mesh import block_tree_mesh
from oracle.operator import PoissonOperator
from oracle.multigrid import MultigridOptions, TreeGeometricMultigrid, jacobi_weight
from oracle.krylov import solve
from oracle import projection as OP
from tpagmg import workloads as W
import reference_cases as RC

GOLD = json.loads((pathlib.Path(__file__).parent / "golden" / "known_answers.json").read_text())


def two_level(bs):
    return block_tree_mesh(block_size=(bs, bs), max_level=2,
                           refine=lambda k, o, e: k[0] == 0 or (k[0] == 1 and k[1] == 0 and k[2] == 0))


@pytest.mark.parametrize("row", GOLD["manufactured_periodic_two_level"]["rows"], ids=lambda r: f"b{r['block']}")
def test_manufactured_errors_match_published_table(row):
    """docs/src/poisson.md:253-257: the L2/Linf errors (4 significant digits)
    pin the composite operator, including the non-diagonal AMR face metric."""
    mesh = two_level(row["block"])
    assert mesh.ncells == row["cells"]
    op = PoissonOperator(mesh)
    mg = TreeGeometricMultigrid(op, MultigridOptions(coarse_size=8))
    x, y = mesh.cell_centers()
    exact = np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y)
    p, st = solve(op, mg, 8 * np.pi ** 2 * exact, rtol=1e-10, max_cycles=60)
    assert st.converged
    v = mesh.cell_volumes()
    err = np.abs(p - exact)
    l2 = np.sqrt(np.sum(v * err ** 2) / np.sum(v))
    assert float(f"{l2:.3e}") == row["l2"]
    assert float(f"{err.max():.3e}") == row["linf"]
    # The PCG column of this hand-written table (8/8/9) is not asserted by the
    # reference's own test (test/operators/poisson.jl:820-831 checks a spread
    # <= 3), and it disagrees with the reference's machine-generated solver
    # checks: the restatement reproduces those exactly on seven solves and four
    # V-cycle spectra (`test_techref_*` below), and takes 9/10/10 here.
    assert st.cycles == {4: 9, 8: 10, 16: 10}[row["block"]]
    assert row["pcg_iterations"] <= st.cycles <= row["pcg_iterations"] + 2


def test_iteration_spread_and_second_order():
    """test/operators/poisson.jl:820-831: spread <= 3, rates > 1.7."""
    res = []
    for bs in (4, 8, 16):
        mesh = two_level(bs)
        op = PoissonOperator(mesh)
        mg = TreeGeometricMultigrid(op, MultigridOptions(coarse_size=8))
        x, y = mesh.cell_centers()
        exact = np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y)
        p, st = solve(op, mg, 8 * np.pi ** 2 * exact, rtol=1e-10, max_cycles=60)
        v = mesh.cell_volumes()
        err = np.abs(p - exact)
        res.append((st.cycles, np.sqrt(np.sum(v * err ** 2) / np.sum(v)), err.max()))
    cycles = [r[0] for r in res]
    assert max(cycles) - min(cycles) <= 3
    for k in (1, 2):
        e = np.array([r[k] for r in res])
        assert np.all(np.diff(e) < 0)
        assert np.min(np.log2(e[:2] / e[1:])) > 1.7


@pytest.mark.parametrize("periodic", [(True, True), (True, False), (False, True), (False, False)])
def test_root_block_hierarchy(periodic):
    g = GOLD["root_block_hierarchy"]
    mesh = block_tree_mesh(base_mesh=tuple(g["base_mesh"]), block_size=tuple(g["block_size"]),
                           origin=(-1.0, 0.25), extent=(2.0, 1.5), periodic=periodic)
    coef = 3.0 + 0.1 * mesh.face_center[:, 0] + 0.2 * mesh.face_center[:, 1] + 0.3 * mesh.face_axis
    op = PoissonOperator(mesh, coef)
    mg = TreeGeometricMultigrid(op, MultigridOptions(coarse_size=g["coarse_size"]))
    assert [list(o.mesh.base_mesh) for o in mg.operators] == g["expected_bases"]
    assert mg.level_sizes == g["expected_sizes"]
    for k, o in enumerate(mg.operators):
        cm = o.mesh
        assert abs(np.sum(o.volumes) - 3.0) <= 128 * np.finfo(float).eps * 3
        expected = 3.0 + 0.1 * cm.face_center[:, 0] + 0.2 * cm.face_center[:, 1] + 0.3 * cm.face_axis
        assert np.allclose(o.face_coefficient, expected, rtol=128 * np.finfo(float).eps, atol=0)
        assert np.max(np.abs(o.matrix @ np.ones(cm.ncells))) <= 1024 * np.finfo(float).eps * max(
            np.max(np.asarray(abs(o.matrix).sum(axis=1))), 1.0)
        for axis in (1, 2):
            tangential = cm.base_mesh[2 - axis]
            assert np.sum(cm.bface_axis == axis) == (0 if periodic[axis - 1] else 2 * tangential)
        if k + 1 < len(mg.operators):
            P = mg.prolongations[k]
            assert np.allclose(P @ np.ones(P.shape[1]), 1.0, atol=128 * np.finfo(float).eps, rtol=0)


@pytest.mark.parametrize("case", GOLD["root_block_hierarchy"]["layout_cases"], ids=str)
def test_isotropic_agglomeration(case):
    layout, expected = case
    mesh = block_tree_mesh(base_mesh=(layout[0] * 4, layout[1] * 4), block_size=(4, 4), periodic=(True, False))
    mg = TreeGeometricMultigrid(PoissonOperator(mesh), MultigridOptions(coarse_size=1))
    assert [list(o.mesh.tree.layout) for o in mg.operators] == expected
    assert mg.level_sizes == [16 * r[0] * r[1] for r in expected]


@pytest.mark.parametrize("case", GOLD["root_block_hierarchy"]["stopping_cases"], ids=str)
def test_stopping_rules(case):
    coarse_size, max_levels, expected = case
    mesh = block_tree_mesh(base_mesh=(16, 16), block_size=(4, 4))
    mg = TreeGeometricMultigrid(PoissonOperator(mesh), MultigridOptions(coarse_size=coarse_size, max_levels=max_levels))
    assert mg.level_sizes == expected


def test_mixed_pruning_sizes():
    g = GOLD["root_block_hierarchy"]["mixed_pruning"]
    mesh = block_tree_mesh(base_mesh=(8, 8), block_size=(4, 4), max_level=1,
                           refine=lambda k, o, e: k == (0, 0, 0))
    mg = TreeGeometricMultigrid(PoissonOperator(mesh), MultigridOptions(coarse_size=g["coarse_size"]))
    assert mg.level_sizes == g["sizes"]


@pytest.mark.parametrize("case", GOLD["periodic_floor"]["cases"], ids=str)
def test_periodic_axes_keep_four_cells(case):
    base, periodic, expected = case
    mesh = block_tree_mesh(base_mesh=tuple(base), block_size=(2, 2), periodic=tuple(periodic))
    mg = TreeGeometricMultigrid(PoissonOperator(mesh), MultigridOptions(coarse_size=1))
    assert [list(o.mesh.base_mesh) for o in mg.operators] == expected


def test_jacobi_weight_policies():
    g = GOLD["jacobi_weight"]
    s = g["skip_case"]
    inv, w = jacobi_weight(np.array(s["diagonal"]), np.array(s["row_sums"]),
                           skip_nonpositive=True, clamp=False, zero_weight=0.0)
    assert list(inv) == s["inverse"] and w == s["weight"]
    with pytest.raises(ValueError):
        jacobi_weight(np.array([2.0, 0.0]), np.array([1.0, 0.0]))
    for d, r, expected in g["clamped"]:
        assert jacobi_weight(np.array(d), np.array(r))[1] == expected
    assert jacobi_weight(np.array([2.0]), np.array([0.0]), skip_nonpositive=True,
                         clamp=False, zero_weight=0.0)[1] == 0.0


def test_factorized_action_matches_assembled_and_nullspace():
    """test/operators/poisson.jl:255-298 and :758-818 (symmetry, A*1 = 0)."""
    mesh = two_level(4)
    coef = 1 + 0.3 * np.sin(np.arange(mesh.nfaces) + 1.0)
    op = PoissonOperator(mesh, coef)
    x = np.sin(0.7 * (np.arange(mesh.ncells) + 1))
    y = np.cos(0.3 * (np.arange(mesh.ncells) + 1))
    ax = op.apply(x)
    assert np.allclose(ax, op.matrix @ x, rtol=64 * np.finfo(float).eps, atol=64 * np.finfo(float).eps * 10)
    assert abs(x @ op.apply(y) - ax @ y) <= 128 * np.finfo(float).eps * abs(ax @ y) + 1e-14
    assert np.max(np.abs(op.apply(np.ones(mesh.ncells)))) <= 64 * np.finfo(float).eps * 10
    w = np.linalg.eigvalsh(op.matrix.toarray())
    tol = 5e-12 * w.max()
    assert w[0] >= -tol and np.sum(np.abs(w) <= tol) == 1


def test_block_partition_independence():
    """test/operators/poisson.jl:884-919: one block, four blocks and four roots
    give the same solution to 2e-12."""
    meshes = [block_tree_mesh(block_size=(16, 16)),
              block_tree_mesh(block_size=(8, 8), max_level=1, refine=lambda k, o, e: True),
              block_tree_mesh(base_mesh=(16, 16), block_size=(8, 8))]
    sols = []
    for mesh in meshes:
        op = PoissonOperator(mesh)
        mg = TreeGeometricMultigrid(op, MultigridOptions(coarse_size=8))
        x, y = mesh.cell_centers()
        p, st = solve(op, mg, 8 * np.pi ** 2 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y), rtol=2e-12)
        assert st.converged
        sols.append(dict(zip(zip(np.round(x, 12), np.round(y, 12)), p)))
    for other in sols[1:]:
        assert other.keys() == sols[0].keys()
        assert max(abs(other[k] - sols[0][k]) for k in sols[0]) <= 2e-12


def test_periodic_nullspace_convention():
    """test/operators/poisson.jl:921-933."""
    mesh = block_tree_mesh(block_size=(8, 8))
    op = PoissonOperator(mesh)
    mg = TreeGeometricMultigrid(op, MultigridOptions(coarse_size=4))
    rhs = np.full(mesh.ncells, 3.0)
    with pytest.raises(ValueError):
        solve(op, mg, rhs, compatibility="error")
    with pytest.raises(ValueError):
        solve(op, mg, rhs, compatibility="invalid")
    p, st = solve(op, mg, rhs, x0=np.full(mesh.ncells, 7.0))
    assert st.converged
    assert abs(st.removed_rhs_mean - 3) < 1e-12
    assert abs(np.sum(p * op.volumes)) <= 16 * np.finfo(float).eps
    assert np.max(np.abs(p)) <= 16 * np.finfo(float).eps


def test_root_block_vcycle_cg_comparison():
    """test/operators/poisson.jl:672-720: capping the hierarchy at four levels
    leaves the 8x8-cell root level as the coarsest (five levels uncapped, down
    to a single 4x4 block); both CG solves of the manufactured field converge
    at rtol 1e-8 to within 1e-6 of it, the uncapped one in no more cycles."""
    from reference_cases import chain_exact, chain_spec
    mesh = block_tree_mesh(**chain_spec())
    op = PoissonOperator(mesh)
    capped = TreeGeometricMultigrid(op, MultigridOptions(coarse_size=16, max_levels=4, pre_sweeps=4, post_sweeps=4))
    full = TreeGeometricMultigrid(op, MultigridOptions(coarse_size=16, pre_sweeps=4, post_sweeps=4))
    assert len(capped.level_sizes) == 4 and len(full.level_sizes) == 5
    assert capped.level_sizes[-1] == 64 and full.level_sizes[-1] == 16
    x, y = mesh.cell_centers()
    exact = chain_exact(x, y)
    rhs = op.apply(exact) / op.volumes  # `apply!`: the strong form
    exact = exact - np.dot(op.volumes, exact) / np.sum(op.volumes)
    (p0, s0), (p1, s1) = (solve(op, mg, rhs, rtol=1e-8, max_cycles=100) for mg in (capped, full))
    assert s0.converged and s1.converged
    assert s0.cycles > 1 and s1.cycles <= s0.cycles
    assert np.max(np.abs(p0 - exact)) <= 1e-6 and np.max(np.abs(p1 - exact)) <= 1e-6


def test_variable_coefficient_operator():
    """test/operators/poisson.jl:788-818: harmonic face means of a 1 / 25 cell
    field lie in [1, 25]; the strong-form action equals minus the divergence of
    the weighted gradient (atol 2e-11, rtol 2e-13); symmetric, positive
    semi-definite with one zero eigenvalue."""
    from oracle import projection as OP
    from reference_cases import harmonic_face_coefficients, two_level_spec
    mesh = block_tree_mesh(**two_level_spec(4))
    cx, cy = mesh.cell_centers()
    kappa = harmonic_face_coefficients(mesh, np.where(cx < 0.5, 1.0, 25.0))
    assert np.all(kappa > 0) and kappa.min() >= 1 and kappa.max() <= 25
    op = PoissonOperator(mesh, kappa)
    p = np.sin(2 * np.pi * cx) * np.cos(2 * np.pi * cy)
    applied = op.apply(p) / op.volumes
    g, gb = OP.weighted_gradient(op, p)
    div = OP.divergence(mesh, g, gb)
    assert np.allclose(applied, -div, atol=2e-11, rtol=2e-13)
    dense = op.matrix.toarray()
    assert np.allclose(dense, dense.T, atol=2e-13, rtol=2e-13)
    w = np.linalg.eigvalsh(dense)
    tol = 5e-12 * w.max()
    assert w[0] >= -tol and np.sum(np.abs(w) <= tol) == 1


def test_preconditioned_and_plain_cg():
    """test/operators/poisson.jl:833-882: on a tree refined to level 4 the
    preconditioned CG (coarse_size 32) converges at rtol 1e-10, and plain CG
    (rtol 1e-8, 500 cycles) converges in more cycles."""
    from reference_cases import deep_rhs, deep_spec
    mesh = block_tree_mesh(**deep_spec())
    op = PoissonOperator(mesh)
    x, y = mesh.cell_centers()
    rhs = deep_rhs(x, y)
    p, st = solve(op, TreeGeometricMultigrid(op, MultigridOptions(coarse_size=32)), rhs, rtol=1e-10, max_cycles=100)
    assert st.converged
    q, plain = solve(op, None, rhs, rtol=1e-8, max_cycles=500, preconditioner=False)
    assert plain.converged and plain.preconditioner == "none"
    assert st.cycles < plain.cycles


class _ComponentLevel:
    """The level data the multigrid component projections read: per-cell
    component slots (-1: inactive), volumes and per-component volumes."""

    def __init__(self, slots, volumes, component_volumes):
        self.slots = slots
        self.volumes = volumes
        self.component_volumes = component_volumes


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("n", [19, 4 * 1024 + 17])
def test_multigrid_component_projections(dtype, n):
    """test/operators/poisson.jl:1245-1357: `_multigrid_remove_component_means!`
    and `_multigrid_project_component_rhs!` on interleaved components with
    inactive cells: the expected projections to 64 eps, zero component sums,
    idempotence, Q and Q' adjoint (256 eps), inactive entries (also non-finite
    ones) untouched, and nothing done on a completely inactive level."""
    from oracle.multigrid import Level
    eps = np.finfo(dtype).eps
    cells = np.arange(1, n + 1)
    index = np.where(cells == n, 4, np.where(cells % 17 == 0, 0, (cells - 1) % 3 + 1))
    volumes = np.where(index == 0, 0, (1 + (5 * cells) % 7) / 8).astype(dtype)
    groups = [np.nonzero(index == c)[0] for c in range(1, 5)]
    inactive = np.nonzero(index == 0)[0]
    active = np.nonzero(index != 0)[0]
    level = _ComponentLevel(index - 1, volumes, np.array([volumes[g].sum() for g in groups], dtype=dtype))
    solution = (((7 * cells) % 31 - 13) / 8).astype(dtype)
    rhs = (((11 * cells) % 37 - 17) / 16).astype(dtype)
    exp_x, exp_b = solution.copy(), rhs.copy()
    for g in groups:
        vol = volumes[g].sum()
        exp_x[g] -= np.dot(volumes[g], solution[g]) / vol
        exp_b[g] -= volumes[g] * (rhs[g].sum() / vol)
    remove = lambda v: Level.remove_means(level, v)  # noqa: E731
    project = lambda v: Level.project_rhs(level, v)  # noqa: E731
    px, pb = remove(solution.copy()), project(rhs.copy())
    tol = 64 * eps
    assert np.allclose(px, exp_x, rtol=tol, atol=tol) and np.allclose(pb, exp_b, rtol=tol, atol=tol)
    assert np.array_equal(px[inactive], solution[inactive]) and np.array_equal(pb[inactive], rhs[inactive])
    for g in groups:
        assert abs(np.dot(volumes[g], px[g])) <= tol * max(np.sum(np.abs(volumes[g] * solution[g])), 1)
        assert abs(np.sum(pb[g])) <= tol * max(np.sum(np.abs(rhs[g])), 1)
    assert np.allclose(remove(px.copy()), px, rtol=tol, atol=tol)
    assert np.allclose(project(pb.copy()), pb, rtol=tol, atol=tol)
    big = 256 * eps * max(np.sqrt(float(np.dot(solution, solution)) * float(np.dot(rhs, rhs))), 1)
    assert np.isclose(np.dot(px, rhs), np.dot(solution, pb), rtol=256 * eps, atol=big)
    normal_x = project(px.copy())
    normal_b = project(remove(rhs.copy()))
    assert np.isclose(np.dot(solution, normal_b), np.dot(rhs, normal_x), rtol=256 * eps, atol=big)
    assert np.isclose(np.dot(solution, normal_x), np.dot(px, px), rtol=256 * eps, atol=big)
    assert np.dot(solution, normal_x) > 0
    # covered entries are neither read nor overwritten
    sentinels = [dtype(np.nan), dtype(np.inf), dtype(-np.inf), dtype(-0.0)]
    for fn, source, expected in ((remove, solution, px), (project, rhs, pb)):
        v = source.copy()
        v[inactive] = [sentinels[k % 4] for k in range(len(inactive))]
        out = fn(v.copy())
        assert np.array_equal(out[inactive], v[inactive], equal_nan=True)
        assert np.array_equal(np.signbit(out[inactive]), np.signbit(v[inactive]))
        assert np.allclose(out[active], expected[active], rtol=tol, atol=tol)
    # a completely inactive level has nothing to normalise
    empty = _ComponentLevel(np.full(n, -1), np.zeros(n, dtype=dtype), np.zeros(0, dtype=dtype))
    v = solution.copy()
    v[0] = np.nan
    for fn in (Level.remove_means, Level.project_rhs):
        assert np.array_equal(fn(empty, v.copy()), v, equal_nan=True)


TECH = GOLD["techref_pressure_solves"]


def techref_operator(maker, n, drop):
    """A fixture of the reference's Chapter 11 solver checks: the mesh and the
    operator (kappa = 1, or 1/rho_f of the drop's mixture density)."""
    mesh = block_tree_mesh(**maker(n))
    if drop:
        frac = W.circle_fractions(mesh, RC.TECHREF_CENTRE, RC.TECHREF_RADIUS)
        _, cond = OP.conditional_fraction(frac)
        return mesh, PoissonOperator(mesh, OP.face_coefficients(mesh, cond, RC.TECHREF_DENSITY))
    return mesh, PoissonOperator(mesh)


@pytest.mark.parametrize("name", list(RC.TECHREF_CASES))
def test_techref_preconditioned_solves(name):
    """`solv_poisson` (docs/techref/figures/solvers.jl:72-93) on the cases of
    `solv_pressure_cases` (:95-113): unknowns, levels, PCG iterations and the
    convergence factor (final_l2 / initial_l2)^(1/cycles) that the reference's
    own run wrote into checks.tex (chkSolv*Cycles/Factor/Levels/Unknowns).
    These pin the V-cycle and the Krylov loop with its strong-residual stop."""
    ref = TECH["solves"][name]
    mesh, op = techref_operator(*RC.TECHREF_CASES[name])
    mg = TreeGeometricMultigrid(op, MultigridOptions())
    _, st = solve(op, mg, RC.techref_noise(mesh.ncells), rtol=1e-10, max_cycles=20000)
    assert st.converged
    assert mesh.ncells == ref["unknowns"]
    assert len(mg.levels) == ref["levels"]
    assert st.cycles == ref["cycles"]
    factor = (st.final_l2 / st.initial_l2) ** (1.0 / st.cycles)
    assert f"{factor:.2f}" == ref["factor"]
    assert f"{mg.levels[0].weight:.3f}" == TECH["omega_uniform128"]


@pytest.mark.parametrize("name", ["uniform64", "uniform128", "amr32", "amr64", "drop128"])
def test_techref_plain_cg(name):
    """The same solves without a preconditioner (chkSolv*Plain): the restated
    Krylov.jl `cg!` recurrence takes exactly the reference's iteration counts
    on the constant-coefficient cases.  At density ratio 1000 thousands of
    unpreconditioned iterations amplify rounding (dot-product order, the
    circle fractions to 1e-10), so the count agrees to 1 %."""
    ref = TECH["solves"][name]
    mesh, op = techref_operator(*RC.TECHREF_CASES[name])
    _, st = solve(op, None, RC.techref_noise(mesh.ncells), rtol=1e-10, max_cycles=20000, preconditioner=False)
    assert st.converged
    if name.startswith("drop"):
        assert abs(st.cycles - ref["plain_cycles"]) <= 0.01 * ref["plain_cycles"]
    else:
        assert st.cycles == ref["plain_cycles"]


def test_techref_vcycle_spectra():
    """`solv_vcycle_check` (solvers.jl:117-165): the V-cycle as a matrix B on
    the compatible subspace, the spectrum of L'(Z'BZ)L with Z'AZ = LL', its
    condition number kappa (chkSolvKappa*), the CG bound (sqrt(kappa) - 1) /
    (sqrt(kappa) + 1), the symmetry of B and the PCG count of each case."""
    import scipy.linalg as sl
    lam_min, lam_max = np.inf, 0.0
    for name, case in RC.TECHREF_VCYCLE_CASES.items():
        ref = TECH["vcycle"][name]
        mesh, op = techref_operator(*case)
        mg = TreeGeometricMultigrid(op, MultigridOptions())
        n = mesh.ncells
        B = np.empty((n, n))
        for j in range(n):
            e = np.zeros(n)
            e[j] = 1.0
            B[:, j] = mg.ldiv(e)
        Z = sl.null_space(op.volumes[None, :])
        L = np.linalg.cholesky(Z.T @ op.matrix.toarray() @ Z)
        M = L.T @ (Z.T @ B @ Z) @ L
        lam = np.linalg.eigvalsh((M + M.T) / 2)
        kappa = lam.max() / lam.min()
        assert f"{kappa:.2f}" == ref["kappa"], name
        assert np.max(np.abs(B - B.T)) <= 1e-14 * np.max(np.abs(B))
        if "bound" in ref:
            assert f"{(np.sqrt(kappa) - 1) / (np.sqrt(kappa) + 1):.2f}" == ref["bound"]
        if "cells" in ref:
            assert n == ref["cells"]
        if "cycles" in ref:
            _, st = solve(op, mg, RC.techref_noise(n), rtol=1e-10, max_cycles=20000)
            assert st.cycles == ref["cycles"]
            assert f"{(st.final_l2 / st.initial_l2) ** (1.0 / st.cycles):.2f}" == ref["factor"]
        lam_min, lam_max = min(lam_min, lam.min()), max(lam_max, lam.max())
    # the published extremes also cover an embedded-solid case that is not on
    # this path; the four cases here lie inside them, the drop at the minimum
    assert f"{lam_min:.3f}" == TECH["lambda_min_all"]
    assert lam_max <= float(TECH["lambda_max_all"])
