"""Open (pressure Dirichlet) sides on the B200 against the oracle and the
reference's testsets (test/operators/poisson.jl:935-1076): the operator with
the open-face conductances, non-singular levels (no compatibility projection,
no augmented coarse solve), solves in FP64 and mixed precision, the open-face
gradient, a coefficient refresh that keeps the boundary coefficients, and a
projection whose open faces keep their velocity.

Tolerances as in test_gpu_parity.py: the action to 1e-13 of |A||x|, solutions
to the oracle's to 1e-10 (FP64, both at rtol 1e-12) and 1e-9 (mixed), the
manufactured pressure to 1e-9 (the reference's own bound)."""
import numpy as np
import pytest

from oracle import projection as OP
from oracle.krylov import solve as osolve
from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions as OMG, TreeGeometricMultigrid
from oracle.operator import PoissonOperator as OOp

pytestmark = pytest.mark.gpu

from tpagmg import BlockTreeMesh, EllipticSolver, MultigridOptions, PoissonOperator, solve  # noqa: E402
from tpagmg import projection as P  # noqa: E402
from tpagmg._lib import TPA_ERR_UNSUPPORTED, TpaError  # noqa: E402

# left = ZeroGradientVelocity(), right = Outflow(), bottom = NoSlip(), top = FreeSlip()
BOUNDARY = {"left": "zero_gradient", "right": "outflow", "bottom": "no_slip", "top": "free_slip"}
OPEN_LR = (True, True, False, False)


def spec_935(mixed, periodic):
    return dict(base_mesh=(16, 8), block_size=(4, 4), extent=(2.0, 1.0), periodic=periodic, max_level=1,
                refine=lambda k, o, e: mixed and k[0] == 0 and k[1] == 3)


def build(mixed, periodic, kappa=1.2):
    spec = spec_935(mixed, periodic)
    m = BlockTreeMesh(**spec)
    om = block_tree_mesh(**spec)
    material = 0.8 + 0.2 * om.bface_center[:, 1]
    op = PoissonOperator(m, kappa, velocity_boundary=BOUNDARY, boundary_face_coefficient=material)
    s = EllipticSolver(op, multigrid=MultigridOptions(coarse_size=8))
    oo = OOp(om, kappa, open_sides=OPEN_LR, boundary_coefficient=material)
    x, y = m.cell_centers()
    v = 0.7 + np.sin(np.pi * x / 2) * np.cos(np.pi * y)
    return m, s, oo, v, material


@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("periodic", [(False, False), (False, True)])
def test_open_sides_operator_and_solves(mixed, periodic):
    m, s, oo, v, material = build(mixed, periodic)
    y = s.apply(v)
    scale = abs(oo.matrix) @ np.abs(v)
    assert np.all(np.abs(y - oo.matrix @ v) <= 1e-13 * scale)
    # no level keeps a nullspace: nothing is projected, the coarse solve is plain
    for level in range(len(s.level_sizes())):
        assert s.level_info(level)[2] == 0
    strong = oo.apply(v) / oo.volumes
    for precision, tol in (("fp64", 1e-9), ("mixed", 1e-9)):
        x = np.zeros(m.ncells)
        st = solve(x, s, strong, rtol=1e-11, max_cycles=300, compatibility="error", precision=precision)
        assert st.converged and st.removed_rhs_mean == 0.0
        assert np.allclose(x, v, atol=tol, rtol=tol)
    rhs = np.cos(3 * np.arange(m.ncells))  # a nonzero-mean right-hand side
    po, so = osolve(oo, TreeGeometricMultigrid(oo, OMG(coarse_size=8)), rhs, rtol=1e-12, compatibility="error")
    x = np.zeros(m.ncells)
    st = solve(x, s, rhs, rtol=1e-12, compatibility="error")
    assert st.converged and abs(st.cycles - so.cycles) <= 1
    assert np.max(np.abs(x - po)) <= 1e-10 * np.max(np.abs(po))
    xm = np.zeros(m.ncells)
    assert solve(xm, s, rhs, rtol=1e-10, compatibility="error", precision="mixed").converged
    assert np.max(np.abs(xm - po)) <= 1e-9 * np.max(np.abs(po))


def test_open_face_gradient_and_refresh():
    m, s, oo, v, material = build(True, (False, False))
    g = P.weighted_gradient(v, s)
    gi, gb = OP.weighted_gradient(oo, v)
    assert np.allclose(g.interior, gi, atol=1e-13, rtol=0)
    assert np.allclose(g.boundary, gb, atol=1e-13, rtol=0)
    ax1 = m.bface_axis == 1
    h = m.spacing[m.bface_cell // 16, 0]
    assert np.allclose(g.boundary[ax1], -m.bface_side[ax1] * material[ax1] * v[m.bface_cell[ax1]] / (h[ax1] / 2),
                       atol=1e-12, rtol=0)
    assert np.all(g.boundary[~ax1] == 0)
    # a coefficient refresh keeps the boundary coefficients (on the host path)
    s.refresh(np.full(m.nfaces, 1.7))
    assert s.last_refresh()[0] == "host"
    oo2 = OOp(block_tree_mesh(**spec_935(True, (False, False))), 1.7, open_sides=OPEN_LR,
              boundary_coefficient=material)
    y = s.apply(v)
    assert np.allclose(y, oo2.matrix @ v, atol=1e-12, rtol=1e-12)
    strong = oo2.apply(v) / oo2.volumes
    x = np.zeros(m.ncells)
    assert solve(x, s, strong, rtol=1e-11, max_cycles=300, compatibility="error").converged
    assert np.allclose(x, v, atol=1e-9, rtol=1e-9)


def test_vertical_open_faces_with_periodic_transverse_direction():
    spec = dict(block_size=(8, 4), extent=(3.0, 1.0), periodic=(True, False))
    m = BlockTreeMesh(**spec)
    s = EllipticSolver(PoissonOperator(m, 2.0, velocity_boundary={"bottom": "zero_gradient", "top": "outflow"}))
    g = P.weighted_gradient(np.ones(m.ncells), s)
    assert np.all(g.interior == 0)
    h = m.spacing[m.bface_cell // 32, 1]
    assert np.all(m.bface_axis == 2)
    assert np.allclose(g.boundary, -m.bface_side * 2 / (h / 2), rtol=1e-15)


def test_projection_keeps_open_face_velocity():
    """project! with an open side: the closed faces are made impermeable, the
    open faces keep their velocity, and the result matches the oracle's."""
    import torch
    m, s, oo, v, material = build(True, (False, False))
    rng = np.random.default_rng(8)
    u = rng.standard_normal(m.nfaces)
    ub = rng.standard_normal(m.nboundary_faces)
    mg = TreeGeometricMultigrid(oo, OMG(coarse_size=8))
    ou, oub, op_, _, ost = OP.project(oo, mg, u, ub, np.zeros(m.ncells), 0.1, tolerance=1e-12)
    ud = torch.from_numpy(u.copy()).cuda()
    ubd = torch.from_numpy(ub.copy()).cuda()
    pd = torch.zeros(m.ncells, dtype=torch.float64, device="cuda")
    st = P.project_device(ud, ubd, pd, s, 0.1, tolerance=1e-12)
    assert st.converged and ost.converged
    scale = max(np.max(np.abs(ou)), np.max(np.abs(oub)))
    assert np.max(np.abs(ud.cpu().numpy() - ou)) <= 1e-9 * scale
    assert np.max(np.abs(ubd.cpu().numpy() - oub)) <= 1e-9 * scale
    assert np.max(np.abs(pd.cpu().numpy() - op_)) <= 1e-9 * np.max(np.abs(op_))
    div = OP.divergence(m, ud.cpu().numpy(), ubd.cpu().numpy())
    assert np.max(np.abs(div)) <= 1e-8 * scale / m.spacing.min()


def test_batch_rejects_open_sides():
    from tpagmg import BatchedSolver
    m, s, oo, v, material = build(False, (False, False))
    with pytest.raises(TpaError) as e:
        BatchedSolver([s])
    assert e.value.code == TPA_ERR_UNSUPPORTED


@pytest.mark.parametrize("explicit", [True, False], ids=["explicit_boundary", "extended_boundary"])
def test_adjoint_with_open_sides_matches_finite_differences(explicit):
    """The adjoint with open sides: dJ/drhs and dJ/dkappa (boundary
    coefficients held fixed, as a refresh keeps them) against central
    differences (step 1e-6) of refreshed solves along 8 seeded directions, to
    1e-6 relative plus the floor of the difference quotient."""
    from test_gpu_adjoint import fd_floor
    spec = spec_935(True, (False, False))
    m = BlockTreeMesh(**spec)
    om = block_tree_mesh(**spec)
    kappa = 1.2 * np.exp(0.3 * np.sin(1.3 * np.arange(m.nfaces)))
    material = 0.8 + 0.2 * om.bface_center[:, 1]
    op = PoissonOperator(m, kappa, velocity_boundary=BOUNDARY,
                         boundary_face_coefficient=material if explicit else None)
    s = EllipticSolver(op, multigrid=MultigridOptions(coarse_size=8))
    x, y = m.cell_centers()
    rhs = np.cos(3 * x) * np.sin(2 * y) + 0.3
    target = np.sin(5 * x + y)

    def J(rhs_, kap):
        s.refresh(kap)
        p_ = np.zeros(m.ncells)
        st = solve(p_, s, rhs_, rtol=1e-13, compatibility="error")
        assert st.converged
        return 0.5 * np.sum((p_ - target) ** 2), p_, st.target_linf

    J0, p0, _ = J(rhs, kappa)
    rb, kb, st = s.adjoint(p0, p0 - target, rtol=1e-13)
    assert st.converged
    rng = np.random.default_rng(77)
    h = 1e-6
    for _ in range(8):
        d = rng.standard_normal(m.ncells)
        jp, _, tp = J(rhs + h * d, kappa)
        jm, _, tm = J(rhs - h * d, kappa)
        fd = (jp - jm) / (2 * h)
        assert abs(fd - rb @ d) <= 1e-6 * abs(fd) + fd_floor(J0, h, (tp, tm), rb), (fd, rb @ d)
        dk = rng.standard_normal(m.nfaces) * kappa
        jp, _, tp = J(rhs, kappa + h * dk)
        jm, _, tm = J(rhs, kappa - h * dk)
        fd = (jp - jm) / (2 * h)
        assert abs(fd - kb @ dk) <= 1e-6 * abs(fd) + fd_floor(J0, h, (tp, tm), rb), (fd, kb @ dk)
    s.refresh(kappa)
