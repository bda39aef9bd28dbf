"""The oracle's projection step against the reference's own known answers
(ronaldremmerswaal/TwoPhaseAMR.jl):

test/two_phase/forces.jl:110-158
* the CSF / CGFM jump is sigma * kappa * jump * |f| bit for bit;
* the weighted jump force equals the weighted gradient of the potential
  sigma * kappa * [c > 1/2] (CGFM) or sigma * kappa * c (CSF) to 5e-13;
* a balanced force projects to a velocity below 1e-9 (dt 0.01, tolerance
  1e-11) at density ratios 1 and 1000 on a uniform, a two-level and a
  band-refined tree.  The reference's third mesh is adapted by `adapt!`; here
  the blocks cut by the circle are refined to the same depth instead.

test/operators/poisson.jl:1704-1747 ("pressure projection")
* a sinusoidal velocity on the two-level tree, kappa = 1 or the harmonic face
  mean of a 1 / 100 cell field: converged, initial >= final residual,
  residual_scale 100, final residual / scale <= 1e-11, dt times the final
  divergence equal to the scaled final residual to 8 eps, the divergence
  reduced below 2e-11 of its initial value, the pressure integral <= 2e-12.

test/operators/poisson.jl:1749-1771 ("incremental pressure projection")
* u = -dt G_k p for p = sin 2 pi x cos 2 pi y on one periodic 8x8 block with
  kappa = 1 + cos(2 pi x_f) / 4: the projection (tolerance 1e-13) returns
  |u| < 1e-10 and |p| < 1e-9.

test/operators/poisson.jl:1773-1797 (tolerance validation)
* an unknown compatibility mode, a reference dt of 0.05 (< dt), inf or nan,
  and a tolerance of 0, -eps, 1, inf or nan are argument errors that leave the
  velocity as it was.

test/operators/poisson.jl:1799-1823 ("mixed-level no-permeation projection")
* a walled two-level tree of 4x4 blocks with u = (0.3 + sin cos, -0.2 + cos sin):
  converged, max |div u| <= 1e-8, zero boundary velocity, pressure integral
  <= 2e-11.
"""
import numpy as np
import pytest

from oracle import projection as P
from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions, TreeGeometricMultigrid
from oracle.operator import PoissonOperator

from tpagmg import workloads as W

from reference_cases import harmonic_face_coefficients  # noqa: F401  (also used by the GPU tests)

CENTER, RADIUS = (0.5, 0.5), 0.2


def mesh_of(kind):
    if kind == 1:
        return dict(block_size=(8, 8), max_level=2)
    if kind == 2:
        return dict(block_size=(8, 8), max_level=2,
                    refine=lambda k, o, e: k[0] == 0 or (k[0] == 1 and k[1] == 0 and k[2] == 0))

    def cut(k, o, e):
        # blocks whose box meets the circle line
        dx = max(abs(o[0] + e[0] / 2 - CENTER[0]) - e[0] / 2, 0.0)
        dy = max(abs(o[1] + e[1] / 2 - CENTER[1]) - e[1] / 2, 0.0)
        far = np.hypot(abs(o[0] + e[0] / 2 - CENTER[0]) + e[0] / 2, abs(o[1] + e[1] / 2 - CENTER[1]) + e[1] / 2)
        return np.hypot(dx, dy) <= RADIUS <= far
    return dict(block_size=(8, 8), max_level=2, refine=cut)


@pytest.mark.parametrize("kind", [1, 2, 3])
@pytest.mark.parametrize("ratio", [1.0, 1000.0])
@pytest.mark.parametrize("formulation", ["csf", "cgfm"])
def test_balanced_force_projects_to_rest(kind, ratio, formulation):
    mesh = block_tree_mesh(**mesh_of(kind))
    raw = W.circle_fractions(mesh, CENTER, RADIUS)
    _, cond = P.conditional_fraction(raw)
    kappa = P.face_coefficients(mesh, cond, (ratio, 1.0))
    op = PoissonOperator(mesh, kappa)
    jumps = P.surface_tension_jumps(mesh, cond, 1.0, 5.0, formulation)
    cm, cp = cond[mesh.face_minus], cond[mesh.face_plus]
    jump = (cp - cm) if formulation == "csf" else (cp > 0.5).astype(float) - (cm > 0.5).astype(float)
    expected = np.where(jump == 0, 0.0, 1.0 * 5.0 * jump * mesh.face_area)
    assert np.array_equal(jumps.view(np.uint64), expected.view(np.uint64))
    force, fb = P.weighted_jump_force(op, jumps)
    assert not fb.any()
    potential = 5.0 * (cond if formulation == "csf" else (cond > 0.5).astype(float))
    g, _ = P.weighted_gradient(op, potential)
    assert np.max(np.abs(force - g)) <= 5e-13
    u = force * 0.01
    mg = TreeGeometricMultigrid(op, MultigridOptions())
    u2, ub, p, phi, st = P.project(op, mg, u, None, np.zeros(mesh.ncells), 0.01, tolerance=1e-11)
    assert st.converged and st.compatible
    assert np.max(np.abs(u2)) < 1e-9
    assert np.all(P.face_coefficients(mesh, cond, (ratio, 1.0)) > 0)


def test_projection_removes_divergence_and_accumulates_pressure():
    """A random velocity: after projection the divergence is at the solve
    tolerance, the pressure is the old one plus the increment, and the step
    with an inherited divergence and a shortened dt follows `_projection_rhs!`."""
    mesh = block_tree_mesh(**mesh_of(2))
    rng = np.random.default_rng(7)
    kappa = np.exp(rng.uniform(-1, 1, mesh.nfaces))
    op = PoissonOperator(mesh, kappa)
    mg = TreeGeometricMultigrid(op, MultigridOptions())
    u = rng.standard_normal(mesh.nfaces)
    p0 = rng.standard_normal(mesh.ncells)
    dt = 0.05
    u2, ub, p, phi, st = P.project(op, mg, u, None, p0, dt, tolerance=1e-10)
    assert st.converged and st.residual_scale == 1 / dt ** 2
    div = P.divergence(mesh, u2, ub)
    assert np.max(np.abs(div)) * dt <= 1e-9
    assert np.array_equal(p, p0 + phi)
    inh = rng.standard_normal(mesh.ncells)
    rhs = P.projection_rhs(P.divergence(mesh, u, ub), dt, inh, 0.08)
    w = (0.08 - dt) / (dt * 0.08)
    assert np.array_equal(rhs, -P.divergence(mesh, u, ub) / dt + w * inh)


def test_conditional_fraction_floor_and_bounds():
    f = np.array([-1e-14, 0.0, 1e-9, 0.3, 1 - 1e-9, 1.0, 1 + 1e-14])
    value, ratio = P.conditional_fraction(f)
    assert list(ratio) == [0.0, 0.0, 0.0, 0.3, 1.0, 1.0, 1.0]
    assert list(value) == [0.0, 0.0, 0.0, 0.3, 1.0, 1.0, 1.0]
    for bad in (-1e-6, 1.0 + 1e-6, np.nan):
        with pytest.raises(ValueError):
            P.conditional_fraction(np.array([0.5, bad]))


def check_projection_known_answer(stats, u_div0, u_div, pressure, volumes):
    """The assertions of test/operators/poisson.jl:1738-1745."""
    initial = np.max(np.abs(u_div0))
    final = np.max(np.abs(u_div))
    assert stats.converged
    assert stats.initial_linf >= stats.final_linf
    assert abs(stats.residual_scale - 100) <= 1e-12 * 100
    assert stats.final_linf / stats.residual_scale <= 1e-11
    assert abs(0.1 * final - stats.final_linf / stats.residual_scale) <= 8 * np.finfo(float).eps
    assert final <= 2e-11 * initial
    assert abs(np.sum(volumes * pressure)) <= 2e-12


@pytest.mark.parametrize("coefficient", ["one", "harmonic"])
def test_pressure_projection_known_answer(coefficient):
    """Two-level tree of 8x8 blocks, u = (sin 2 pi x cos 2 pi y, cos 2 pi x
    sin 2 pi y) at the face centres, dt 0.1, tolerance 1e-11, coarse_size 8."""
    mesh = block_tree_mesh(**mesh_of(2))
    x, y = mesh.face_center[:, 0], mesh.face_center[:, 1]
    u0 = np.where(mesh.face_axis == 1, np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y),
                  np.cos(2 * np.pi * x) * np.sin(2 * np.pi * y))
    if coefficient == "one":
        kappa = np.ones(mesh.nfaces)
    else:
        cx, _ = mesh.cell_centers()
        kappa = harmonic_face_coefficients(mesh, np.where(cx < 0.5, 1.0, 100.0))
    op = PoissonOperator(mesh, kappa)
    mg = TreeGeometricMultigrid(op, MultigridOptions(coarse_size=8))
    u, ub, p, phi, st = P.project(op, mg, u0, None, np.zeros(mesh.ncells), 0.1, tolerance=1e-11)
    check_projection_known_answer(st.solve, P.divergence(mesh, u0, ub), P.divergence(mesh, u, ub), p,
                                  mesh.cell_volumes())


def incremental_case(mesh):
    """Coefficients and the velocity -dt G_k p of test/operators/poisson.jl:1749-1762."""
    kappa = 1 + 0.25 * np.cos(2 * np.pi * mesh.face_center[:, 0])
    x, y = mesh.cell_centers()
    return kappa, np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y)


def test_incremental_pressure_projection_known_answer():
    mesh = block_tree_mesh(block_size=(8, 8))
    kappa, p0 = incremental_case(mesh)
    op = PoissonOperator(mesh, kappa)
    g, _ = P.weighted_gradient(op, p0)
    u0 = -0.1 * g
    mg = TreeGeometricMultigrid(op, MultigridOptions(coarse_size=8))
    u, ub, p, phi, st = P.project(op, mg, u0, None, p0, 0.1, tolerance=1e-13, max_cycles=100)
    assert st.converged
    assert np.max(np.abs(u)) < 1e-10
    assert np.max(np.abs(p)) < 1e-9


def test_projection_argument_validation():
    mesh = block_tree_mesh(block_size=(4, 4))
    op = PoissonOperator(mesh)
    mg = TreeGeometricMultigrid(op, MultigridOptions(coarse_size=4))
    u = np.ones(mesh.nfaces)
    original = u.copy()
    with pytest.raises(ValueError):
        P.project(op, mg, u, None, np.zeros(mesh.ncells), 0.1, compatibility="invalid")
    for bad in (0.05, np.inf, np.nan):
        with pytest.raises(ValueError):
            P.project(op, mg, u, None, np.zeros(mesh.ncells), 0.1, reference_dt=bad)
    for bad in (0.0, -np.finfo(float).eps, 1.0, np.inf, np.nan):
        with pytest.raises(ValueError):
            P.project(op, mg, u, None, np.zeros(mesh.ncells), 0.1, tolerance=bad)
    assert np.array_equal(u, original)


def no_permeation_case():
    """Mesh and velocity of test/operators/poisson.jl:1799-1811."""
    spec = dict(block_size=(4, 4), periodic=(False, False), max_level=2,
                refine=lambda k, o, e: k[0] == 0 or (k[0] == 1 and k[1] == 0 and k[2] == 0))
    mesh = block_tree_mesh(**spec)

    def field(center, axis):
        x, y = center[:, 0], center[:, 1]
        return np.where(axis == 1, 0.3 + np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y),
                        -0.2 + np.cos(2 * np.pi * x) * np.sin(2 * np.pi * y))
    return spec, mesh, field(mesh.face_center, mesh.face_axis), field(mesh.bface_center, mesh.bface_axis)


def test_mixed_level_no_permeation_projection_known_answer():
    _, mesh, u0, ub0 = no_permeation_case()
    assert len(ub0) > 0 and np.any(ub0)
    op = PoissonOperator(mesh)
    mg = TreeGeometricMultigrid(op, MultigridOptions(coarse_size=8))
    u, ub, p, phi, st = P.project(op, mg, u0, ub0, np.zeros(mesh.ncells), 0.05, tolerance=1e-10, max_cycles=80)
    assert st.converged
    assert np.max(np.abs(P.divergence(mesh, u, ub))) <= 1e-8
    assert not np.any(ub)
    assert abs(np.sum(mesh.cell_volumes() * p)) <= 2e-11
