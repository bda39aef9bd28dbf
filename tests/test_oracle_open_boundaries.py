"""Open (pressure Dirichlet) sides in the oracle, against the reference's
testsets "open pressure boundary operators and solvers" and "vertical open
pressure faces with periodic transverse direction" (test/operators/
poisson.jl:935-1076).  An open side (Outflow or ZeroGradientVelocity of the
velocity) adds the conductance 2 k_b / h |f| of its faces to the diagonal,
anchors the components it touches (no nullspace, no compatibility
projection) and gives the faces the gradient -side k_b p / (h / 2)."""
import numpy as np
import pytest

from oracle import projection as OP
from oracle.krylov import solve
from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions, TreeGeometricMultigrid
from oracle.operator import PoissonOperator

# left = ZeroGradientVelocity(), right = Outflow(), bottom = NoSlip(), top = FreeSlip()
OPEN_LR = (True, True, False, False)


def mesh_935(mixed, periodic):
    return block_tree_mesh(base_mesh=(16, 8), block_size=(4, 4), extent=(2.0, 1.0), periodic=periodic,
                           max_level=1, refine=lambda k, o, e: mixed and k[0] == 0 and k[1] == 3)


def pressure_935(mesh):
    x, y = mesh.cell_centers()
    return 0.7 + np.sin(np.pi * x / 2) * np.cos(np.pi * y)


@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("periodic", [(False, False), (False, True)])
def test_open_pressure_boundary_operators_and_solvers(mixed, periodic):
    mesh = mesh_935(mixed, periodic)
    material = 0.8 + 0.2 * mesh.bface_center[:, 1]
    op = PoissonOperator(mesh, 1.2, open_sides=OPEN_LR, boundary_coefficient=material)
    assert not op.singular
    v = pressure_935(mesh)
    # the factorized action and the assembled matrix
    assert np.allclose(op.apply(v), op.matrix @ v, atol=1e-12, rtol=1e-12)
    # interior coefficients extended to the open faces of axis 1
    ext = PoissonOperator(mesh, np.full(mesh.nfaces, 1.2), open_sides=OPEN_LR)
    ax1 = mesh.bface_axis == 1
    assert np.allclose(ext.boundary_coefficient[ax1], 1.2, rtol=1e-15)
    # weighted gradient, its divergence and the open-face gradient
    g = op.weighted_gradient(v)
    gb = op.boundary_weighted_gradient(v)
    strong = op.apply(v) / op.volumes
    assert np.allclose(strong, -OP.divergence(mesh, g, gb), atol=2e-12, rtol=0)
    nx, ny = mesh.block_size
    h = mesh.spacing[mesh.bface_cell // (nx * ny), 0]
    expected = -mesh.bface_side * material * v[mesh.bface_cell] / (h / 2)
    assert np.allclose(gb[ax1], expected[ax1], atol=1e-12, rtol=0)
    assert np.all(gb[~ax1] == 0)
    # a nonzero-mean RHS is solved without a compatibility projection, and the
    # coarse solve is not augmented (no level is singular)
    mg = TreeGeometricMultigrid(op, MultigridOptions(coarse_size=8))
    assert all(not o.singular for o in mg.operators)
    assert mg.coarse_matrix.shape[0] == mg.levels[-1].n
    p, st = solve(op, mg, strong, rtol=1e-11, max_cycles=300, compatibility="error")
    assert st.converged and st.removed_rhs_mean == 0.0
    assert np.allclose(p, v, atol=1e-9, rtol=1e-9)
    # a coefficient refresh keeps the boundary diagonal on every level
    op.update_boundary_coefficient(np.full(len(mesh.bface_cell), 0.6))
    mg.refresh(np.full(mesh.nfaces, 1.7))
    assert all(not o.singular for o in mg.operators)
    for o in mg.operators:
        sel = o.mesh.bface_axis == 1
        assert np.allclose(o.boundary_coefficient[sel], 0.6, rtol=1e-15)
    strong = op.apply(v) / op.volumes
    p, st = solve(op, mg, strong, rtol=1e-11, max_cycles=300, compatibility="error")
    assert st.converged and np.allclose(p, v, atol=1e-9, rtol=1e-9)


def test_vertical_open_faces_with_periodic_transverse_direction():
    mesh = block_tree_mesh(block_size=(8, 4), extent=(3.0, 1.0), periodic=(True, False))
    op = PoissonOperator(mesh, 2.0, open_sides=(False, False, True, True))
    p = np.ones(mesh.ncells)
    assert np.all(op.weighted_gradient(p) == 0)
    gb = op.boundary_weighted_gradient(p)
    nx, ny = mesh.block_size
    assert np.all(mesh.bface_axis == 2)
    h = mesh.spacing[mesh.bface_cell // (nx * ny), 1]
    assert np.allclose(gb, -mesh.bface_side * 2 / (h / 2), rtol=1e-15)
    strong = op.apply(p) / op.volumes
    assert np.allclose(strong, -OP.divergence(mesh, op.weighted_gradient(p), gb), atol=1e-12, rtol=0)


def test_opposite_open_faces_need_boundary_material():
    """test/operators/poisson.jl:1143-1158: on a one-cell column (no interior
    face; a topology a mesh cannot have, built here as the reference builds
    it), a scalar coefficient fills both open faces, and a vector of interior
    coefficients cannot be extended to them."""
    from types import SimpleNamespace
    from oracle.operator import boundary_material
    column = SimpleNamespace(nfaces=0, face_minus=np.zeros(0, int), face_plus=np.zeros(0, int),
                             face_axis=np.zeros(0, int), face_area=np.zeros(0),
                             bface_cell=np.array([0, 0]), bface_axis=np.array([1, 1]),
                             bface_side=np.array([-1, 1]), bface_area=np.array([1.0, 1.0]))
    assert list(boundary_material(column, 2.5, OPEN_LR)) == [2.5, 2.5]
    with pytest.raises(ValueError):
        boundary_material(column, np.zeros(0), OPEN_LR)
