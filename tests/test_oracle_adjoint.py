"""The oracle's adjoint of the pressure solve, pinned on the CPU against
central finite differences of the loss through exact (direct) solves.

The reference differentiates nothing, so the adjoint is pinned by the
definition of the derivative: J = 1/2 ||p - p_t||^2 over a disk of cells, p
from the gauged, projected solve of `solve!` (elliptic_solver.jl:628-675), and
central differences with step 1e-6 along seeded random directions of the
strong right-hand side and of the face coefficients.
"""
import numpy as np
import pytest

from oracle.adjoint import adjoint, exact_solve, face_gradient, loss, loss_cotangent, loss_mask
from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions, TreeGeometricMultigrid
from oracle.operator import PoissonOperator


def two_level(bs):
    return dict(block_size=(bs, bs), max_level=2,
                refine=lambda k, o, e: k[0] == 0 or (k[0] == 1 and k[1] == 0 and k[2] == 0))


def problem(seed=3):
    mesh = block_tree_mesh(**two_level(4))
    rng = np.random.default_rng(seed)
    kappa = np.exp(0.5 * rng.standard_normal(mesh.nfaces))
    op = PoissonOperator(mesh, kappa)
    x, y = mesh.cell_centers()
    f = rng.standard_normal(mesh.ncells)
    target = rng.standard_normal(mesh.ncells)
    mask = loss_mask((x, y), center=(0.5, 0.5), radius=0.3)
    return mesh, op, f, target, mask


def fd_roundoff(J0, h):
    """Rounding floor of a central difference of J with step h."""
    return 64 * np.finfo(np.float64).eps * max(abs(J0), 1.0) / h


def J_of(op, f, target, mask):
    return loss(exact_solve(op, f), target, mask)


def test_problem_has_hanging_vertex_patches():
    mesh, op, *_ = problem()
    assert not op.diagonal_metric
    assert op.K.nnz > mesh.nfaces


def test_rhs_gradient_matches_central_differences():
    mesh, op, f, target, mask = problem()
    p = exact_solve(op, f)
    rhs_bar, _, _ = adjoint(op, p, loss_cotangent(p, target, mask), exact=True)
    J0 = loss(p, target, mask)
    rng = np.random.default_rng(505)
    h = 1e-6
    for _ in range(8):
        d = rng.standard_normal(mesh.ncells)
        fd = (J_of(op, f + h * d, target, mask) - J_of(op, f - h * d, target, mask)) / (2 * h)
        assert abs(fd - rhs_bar @ d) <= 1e-6 * abs(fd) + fd_roundoff(J0, h)


def test_face_coefficient_gradient_matches_central_differences():
    mesh, op, f, target, mask = problem()
    p = exact_solve(op, f)
    _, kappa_bar, _ = adjoint(op, p, loss_cotangent(p, target, mask), exact=True)
    J0 = loss(p, target, mask)
    kappa = op.face_coefficient.copy()
    metric = (op.K, op.diagonal_metric, op.metric_templates)
    rng = np.random.default_rng(506)
    h = 1e-6
    for _ in range(8):
        d = rng.standard_normal(mesh.nfaces) * kappa
        jp = J_of(PoissonOperator(mesh, kappa + h * d, metric=metric), f, target, mask)
        jm = J_of(PoissonOperator(mesh, kappa - h * d, metric=metric), f, target, mask)
        fd = (jp - jm) / (2 * h)
        assert abs(fd - kappa_bar @ d) <= 1e-6 * abs(fd) + fd_roundoff(J0, h)


def test_krylov_adjoint_matches_exact_adjoint():
    mesh, op, f, target, mask = problem()
    p = exact_solve(op, f)
    pbar = loss_cotangent(p, target, mask)
    mg = TreeGeometricMultigrid(op, MultigridOptions(coarse_size=8))
    rb, kb, lam = adjoint(op, p, pbar, mg, rtol=1e-13)
    rbe, kbe, lame = adjoint(op, p, pbar, exact=True)
    assert np.max(np.abs(lam - lame)) <= 1e-10 * np.max(np.abs(lame))
    assert np.max(np.abs(rb - rbe)) <= 1e-10 * np.max(np.abs(rbe))
    assert np.max(np.abs(kb - kbe)) <= 1e-9 * np.max(np.abs(kbe))


def test_face_gradient_is_bilinear_and_diagonal_rows_are_products():
    mesh, op, f, target, mask = problem()
    rng = np.random.default_rng(9)
    p, q, lam = (rng.standard_normal(mesh.ncells) for _ in range(3))
    g = face_gradient(op, p + 2 * q, lam)
    assert np.allclose(g, face_gradient(op, p, lam) + 2 * face_gradient(op, q, lam), rtol=1e-12, atol=1e-12)
    diag_rows = np.asarray((op.K != 0).sum(axis=1)).ravel() == 1
    u, w = op.J @ p, op.J @ lam
    assert np.any(diag_rows)
    np.testing.assert_allclose(face_gradient(op, p, lam)[diag_rows], -(op.K.diagonal() * u * w)[diag_rows],
                               rtol=1e-14, atol=0)


def test_symmetric_gradient_of_quadratic_form():
    """dS/dkappa_f is symmetric, so lam'(dS/dkappa_f)p = p'(dS/dkappa_f)lam."""
    mesh, op, *_ = problem()
    rng = np.random.default_rng(12)
    p, lam = rng.standard_normal(mesh.ncells), rng.standard_normal(mesh.ncells)
    np.testing.assert_allclose(face_gradient(op, p, lam), face_gradient(op, lam, p), rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("seed", [1, 2])
def test_exact_solve_is_gauged_and_solves(seed):
    mesh, op, f, *_ = problem(seed)
    p = exact_solve(op, f)
    v = op.volumes
    assert abs(np.dot(v, p)) <= 1e-12 * np.sum(v) * np.max(np.abs(p))
    b = f * v
    b -= v * b.sum() / v.sum()
    assert np.max(np.abs(op.matrix @ p - b)) <= 1e-11 * np.max(np.abs(b))
