"""The lattice addressing of the row-streaming kernels (csrc/stream.cuh), on
the CPU, against the oracle's hierarchy.

The kernels address a cell of a periodic single-level lattice by its lattice
position alone: block (gx / 16, gy / 16) in row-major order, then the row-major
cell inside the 16 x 16 block (`st_cell`); the next level's cell holding it is
the same formula at (gx / 2, gy / 2) on the halved lattice (`st_coarse`).  The
host admits a level only when its keys, neighbour table and block map say so
(`stream_lattice` in csrc/solve_fused.cu).  Here the formulas are checked
against the oracle's restated meshes (the reference's (level, j, i) block sort,
mesh/topology/mesh.jl:1059-1121) and its tentative-transfer owners
(tree_coarsening.jl:228-252), and the library's owners against both."""
import numpy as np
import pytest

from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions as OMG, TreeGeometricMultigrid
from oracle.operator import PoissonOperator as OOp

from tpagmg import BlockTreeMesh, EllipticSolver, MultigridOptions, PoissonOperator  # noqa: E402


def st_cell(nbx, gx, gy):
    return (((gy >> 4) * nbx + (gx >> 4)) << 8) + ((gy & 15) << 4) + (gx & 15)


def st_coarse(nbx, gx, gy):
    cx, cy = gx >> 1, gy >> 1
    return (((cy >> 4) * (nbx >> 1) + (cx >> 4)) << 8) + ((cy & 15) << 4) + (cx & 15)


def lattice(keys):
    """(nbx, nby) when the keys are one level filling a rectangle in row-major
    order, else None (the host's admission rule for the keys)."""
    lev = {k[0] for k in keys}
    if len(lev) != 1:
        return None
    nbx = max(k[1] for k in keys) + 1
    nby = max(k[2] for k in keys) + 1
    if nbx * nby != len(keys):
        return None
    (lv,) = lev
    if any(keys[b] != (lv, b % nbx, b // nbx) for b in range(len(keys))):
        return None
    return nbx, nby


CASES = {
    "periodic_128": dict(base_mesh=(128, 128), block_size=(16, 16), periodic=(True, True)),
    "periodic_256x128": dict(base_mesh=(256, 128), block_size=(16, 16), extent=(2.0, 1.0), periodic=(True, True)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_lattice_formulas_match_the_hierarchy(name):
    spec = CASES[name]
    om = block_tree_mesh(**spec)
    mg = TreeGeometricMultigrid(OOp(om, np.ones(om.nfaces)), OMG(coarse_size=64))
    s = EllipticSolver(PoissonOperator(BlockTreeMesh(**spec)), multigrid=MultigridOptions(coarse_size=64))
    checked = 0
    for lev in range(len(mg.levels) - 1):
        fine, coarse = mg.operators[lev].mesh, mg.operators[lev + 1].mesh
        lat, clat = lattice(fine.keys), lattice(coarse.keys)
        if lat is None or clat is None or lat[0] % 2 or lat[1] % 2 or clat != (lat[0] // 2, lat[1] // 2):
            continue
        nbx, nby = lat
        gy, gx = np.meshgrid(np.arange(16 * nby), np.arange(16 * nbx), indexing="ij")
        gx, gy = gx.ravel(), gy.ravel()
        cells = st_cell(nbx, gx, gy)
        # every cell exactly once
        assert np.array_equal(np.sort(cells), np.arange(16 * 16 * nbx * nby))
        # the cell's lattice position is its geometric position: block origin
        # plus the offset inside the block, one spacing per lattice step
        b, lx, ly = cells >> 8, cells & 15, (cells >> 4) & 15
        hx, hy = fine.spacing[b, 0], fine.spacing[b, 1]
        assert np.allclose(fine.block_origin[b, 0] + (lx + 0.5) * hx, fine.origin[0] + (gx + 0.5) * hx,
                           rtol=0, atol=1e-12)
        assert np.allclose(fine.block_origin[b, 1] + (ly + 0.5) * hy, fine.origin[1] + (gy + 0.5) * hy,
                           rtol=0, atol=1e-12)
        own = mg.owners[lev]
        assert np.array_equal(own[cells], st_coarse(nbx, gx, gy))
        assert np.array_equal(s.level_owners(lev)[cells], st_coarse(nbx, gx, gy))
        # the neighbours the kernels take by wrapping the lattice position are
        # the mesh's periodic faces: x faces join (W - 1, y) and (0, y), y faces
        # (x, H - 1) and (x, 0)
        W, H = 16 * nbx, 16 * nby
        faces = set(zip(fine.face_minus.tolist(), fine.face_plus.tolist(), fine.face_axis.tolist()))
        for y in range(0, H, 7):
            assert (st_cell(nbx, W - 1, y), st_cell(nbx, 0, y), 1) in faces
        for x in range(0, W, 7):
            assert (st_cell(nbx, x, H - 1), st_cell(nbx, x, 0), 2) in faces
        checked += 1
    # every multi-block level of these meshes down to 2 x 2 blocks is a lattice level
    assert checked >= 2


def test_refined_tree_is_not_a_lattice():
    """The key rule turns down a tree with two levels of blocks and admits a
    one-level rectangle."""
    two = block_tree_mesh(base_mesh=(64, 64), block_size=(16, 16), max_level=2,
                          refine=lambda k, o, e: k[0] == 0 and k[1] == 0 and k[2] == 0)
    assert lattice(two.keys) is None
    flat = block_tree_mesh(base_mesh=(64, 32), block_size=(16, 16), extent=(2.0, 1.0), periodic=(True, True))
    assert lattice(flat.keys) == (4, 2)
