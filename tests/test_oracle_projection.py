"""The oracle's projection step against the reference's own known answers
(test/two_phase/forces.jl:110-158 of ronaldremmerswaal/TwoPhaseAMR.jl):

* the CSF / CGFM jump is sigma * kappa * jump * |f| bit for bit;
* the weighted jump force equals the weighted gradient of the potential
  sigma * kappa * [c > 1/2] (CGFM) or sigma * kappa * c (CSF) to 5e-13;
* a balanced force projects to a velocity below 1e-9 (dt 0.01, tolerance
  1e-11) at density ratios 1 and 1000 on a uniform, a two-level and a
  band-refined tree.

The reference's third mesh is adapted by `adapt!`; here the blocks cut by the
circle are refined to the same depth instead.
"""
import numpy as np
import pytest

from oracle import projection as P
from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions, TreeGeometricMultigrid
from oracle.operator import PoissonOperator

from tpagmg import workloads as W

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
