"""The V-cycle on haloed block tiles (two launches per CSR level,
csrc/tiles.cuh) against the unfused kernels and the oracle.

Both layouts run the CSR kernels on every multi-CTA level (structured = 0),
so the only difference is the tiling.  Tolerances: one FP64 V-cycle to 1e-13
of max |z| (the rows are summed in the same order; only the coarse RHS sums
fold their partials in another order), one mixed V-cycle to 1e-5, solutions
to the oracle's to 1e-10 (FP64, rtol 1e-12) and 1e-9 (mixed).
"""
import numpy as np
import pytest

from oracle.krylov import solve as osolve
from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions as OMG, TreeGeometricMultigrid
from oracle.operator import PoissonOperator as OOp

pytestmark = pytest.mark.gpu

from tpagmg import BlockTreeMesh, EllipticSolver, MultigridOptions, PoissonOperator, solve  # noqa: E402
from tpagmg import workloads as W  # noqa: E402
import reference_cases as RC  # noqa: E402


def two_level(bs):
    return dict(block_size=(bs, bs), max_level=2,
                refine=lambda k, o, e: k[0] == 0 or (k[0] == 1 and k[1] == 0 and k[2] == 0))


CASES = {
    "droplet_l2": (W.droplet_spec(levels=2), 64, "droplet"),
    "droplet_l3": (W.droplet_spec(levels=3), 64, "droplet"),
    "two_level_b16": (two_level(16), 8, None),
    "walls_varcoef_b16": (dict(base_mesh=(128, 128), block_size=(16, 16), periodic=(False, False)), 64,
                          lambda m: np.exp(0.5 * np.sin(0.3 * np.arange(m.nfaces)))),
    "periodic_b16": (dict(base_mesh=(128, 64), block_size=(16, 16), extent=(2.0, 1.0), periodic=(True, True)), 64,
                     None),
    "techref_amr32_b8": (RC.techref_amr(32), 64, None),
}


def build(name, tiles):
    spec, coarse, coef = CASES[name]
    m = BlockTreeMesh(**spec)
    if coef == "droplet":
        _, kappa, _ = W.droplet_inputs(m)
    elif coef is None:
        kappa = np.ones(m.nfaces)
    else:
        kappa = coef(m)
    s = EllipticSolver(PoissonOperator(m, kappa), multigrid=MultigridOptions(coarse_size=coarse))
    s.set_tuning(structured=0, tiles=tiles, tail_cells=1024)
    return spec, m, kappa, coarse, s


@pytest.mark.parametrize("name", list(CASES))
def test_tiled_vcycle_matches_unfused(name):
    spec, m, kappa, coarse, s = build(name, 1)
    _, _, _, _, s0 = build(name, 0)
    assert s.tiled_levels() >= 1 and s0.tiled_levels() == 0
    rng = np.random.default_rng(9)
    vol = m.cell_volumes()
    for trial in range(2):  # twice: the tile buffers are reused
        r = rng.standard_normal(m.ncells) * vol
        r -= vol * np.sum(r) / np.sum(vol)
        for precision, tol in (("fp64", 1e-13), ("mixed", 1e-5)):
            z, z0 = s.vcycle(r, precision=precision), s0.vcycle(r, precision=precision)
            assert np.max(np.abs(z - z0)) <= tol * np.max(np.abs(z0)), (precision, trial)


@pytest.mark.parametrize("name", ["droplet_l2", "walls_varcoef_b16", "techref_amr32_b8"])
def test_tiled_solve_matches_oracle(name):
    spec, m, kappa, coarse, s = build(name, 1)
    _, _, _, _, s0 = build(name, 0)
    oo = OOp(block_tree_mesh(**spec), kappa)
    rhs = W.gaussian_rhs(m, 21)
    po, so = osolve(oo, TreeGeometricMultigrid(oo, OMG(coarse_size=coarse)), rhs, rtol=1e-12)
    x, x0 = np.zeros(m.ncells), np.zeros(m.ncells)
    st, st0 = solve(x, s, rhs, rtol=1e-12), solve(x0, s0, rhs, rtol=1e-12)
    assert st.converged and st.cycles == st0.cycles and abs(st.cycles - so.cycles) <= 1
    assert np.max(np.abs(x - po)) <= 1e-10 * np.max(np.abs(po))
    xm = np.zeros(m.ncells)
    stm = solve(xm, s, rhs, rtol=1e-10, precision="mixed")
    assert stm.converged
    assert np.max(np.abs(xm - po)) <= 1e-9 * np.max(np.abs(po))


def test_tiled_refresh_matches_rebuild():
    """A device refresh updates the tile copies of the level values."""
    spec, m, kappa, coarse, s = build("droplet_l2", 1)
    k2 = kappa * (1.0 + 0.2 * np.cos(np.arange(m.nfaces)))
    s.refresh(k2)
    fresh = EllipticSolver(PoissonOperator(m, k2), multigrid=MultigridOptions(coarse_size=coarse))
    fresh.set_tuning(structured=0, tiles=0, tail_cells=1024)
    rng = np.random.default_rng(2)
    vol = m.cell_volumes()
    r = rng.standard_normal(m.ncells) * vol
    r -= vol * np.sum(r) / np.sum(vol)
    z, z0 = s.vcycle(r, precision="fp64"), fresh.vcycle(r, precision="fp64")
    assert np.max(np.abs(z - z0)) <= 1e-12 * np.max(np.abs(z0))


VEC_CASES = {
    "periodic_256": dict(base_mesh=(256, 256), block_size=(16, 16), periodic=(True, True)),
    "walls_128": dict(base_mesh=(128, 128), block_size=(16, 16), periodic=(False, False)),
    "channel_256x128": dict(base_mesh=(256, 128), block_size=(16, 16), extent=(2.0, 1.0), periodic=(True, False)),
}


@pytest.mark.parametrize("name", list(VEC_CASES))
def test_stencil_tiles_match_vectorized_kernels(name):
    """Constant-coefficient 16x16 levels: the 22 x 22 stencil tiles against the
    vectorized six-launch kernels and the oracle."""
    spec = VEC_CASES[name]
    m = BlockTreeMesh(**spec)
    s = EllipticSolver(PoissonOperator(m), multigrid=MultigridOptions(coarse_size=64))
    s0 = EllipticSolver(PoissonOperator(m), multigrid=MultigridOptions(coarse_size=64))
    s.set_tuning(tiles=2, tail_cells=1024)
    s0.set_tuning(tiles=0, tail_cells=1024)
    assert s.device_info()["structured_levels"] >= 1
    assert s.tiled_levels() >= 1 and s0.tiled_levels() == 0
    rng = np.random.default_rng(4)
    vol = m.cell_volumes()
    for trial in range(2):
        r = rng.standard_normal(m.ncells) * vol
        r -= vol * np.sum(r) / np.sum(vol)
        for precision, tol in (("fp64", 1e-13), ("mixed", 1e-5)):
            z, z0 = s.vcycle(r, precision=precision), s0.vcycle(r, precision=precision)
            assert np.max(np.abs(z - z0)) <= tol * np.max(np.abs(z0)), (precision, trial)
    oo = OOp(block_tree_mesh(**spec), np.ones(m.nfaces))
    rhs = W.gaussian_rhs(m, 5)
    po, _ = osolve(oo, TreeGeometricMultigrid(oo, OMG(coarse_size=64)), rhs, rtol=1e-12)
    x, xm = np.zeros(m.ncells), np.zeros(m.ncells)
    assert solve(x, s, rhs, rtol=1e-12).converged
    assert solve(xm, s, rhs, rtol=1e-10, precision="mixed").converged
    assert np.max(np.abs(x - po)) <= 1e-10 * np.max(np.abs(po))
    assert np.max(np.abs(xm - po)) <= 1e-9 * np.max(np.abs(po))


def test_stencil_tiles_on_small_levels_only():
    """tiles = 3: stencil tiles on the constant-coefficient levels of at most
    2^19 cells; the 1024^2 finest level keeps the vectorized kernels.  The
    V-cycle equals the six-launch one to rounding, and the solve reaches the
    tolerance in the same number of iterations."""
    m = BlockTreeMesh(base_mesh=(1024, 1024), block_size=(16, 16), periodic=(True, True))
    s = EllipticSolver(PoissonOperator(m))
    s0 = EllipticSolver(PoissonOperator(m))
    s2 = EllipticSolver(PoissonOperator(m))
    s.set_tuning(tiles=3, tail_cells=1024)
    s0.set_tuning(tiles=0, tail_cells=1024)
    s2.set_tuning(tiles=2, tail_cells=1024)
    multi = [n for n in s.level_sizes()[:-1] if n > 1024]  # the levels outside the one-CTA tail
    assert s0.device_info()["structured_levels"] >= len(multi)
    assert s2.tiled_levels() == len(multi)
    assert s.tiled_levels() == sum(1 for n in multi if n <= 1 << 19) == len(multi) - 1
    rng = np.random.default_rng(11)
    r = rng.standard_normal(m.ncells)
    r -= r.mean()
    r *= m.cell_volumes()
    for precision, tol in (("fp64", 1e-13), ("mixed", 1e-5)):
        z, z0 = s.vcycle(r, precision=precision), s0.vcycle(r, precision=precision)
        assert np.max(np.abs(z - z0)) <= tol * np.max(np.abs(z0)), precision
    rhs = r / m.cell_volumes()
    for precision in ("fp64", "mixed"):
        x, x0 = np.zeros(m.ncells), np.zeros(m.ncells)
        st = solve(x, s, rhs, rtol=1e-10, precision=precision)
        st0 = solve(x0, s0, rhs, rtol=1e-10, precision=precision)
        assert st.converged and st0.converged and st.cycles == st0.cycles
        assert np.max(np.abs(x - x0)) <= 1e-9 * np.max(np.abs(x0))


STREAM_CASES = {
    # (mesh, levels expected on the row-streaming kernels with tiles = 5, tail cells)
    "periodic_256": (dict(base_mesh=(256, 256), block_size=(16, 16), periodic=(True, True)), 3, 1024),
    "periodic_256x128": (dict(base_mesh=(256, 128), block_size=(16, 16), extent=(2.0, 1.0),
                              periodic=(True, True)), 3, 1024),
    # down to the 32 x 32 level (2 x 2 blocks, one strip wrapping across it), only
    # the 16 x 16 level in the tail
    "periodic_128_tail256": (dict(base_mesh=(128, 128), block_size=(16, 16), periodic=(True, True)), 3, 256),
    "channel_256x128": (dict(base_mesh=(256, 128), block_size=(16, 16), extent=(2.0, 1.0),
                             periodic=(True, False)), 0, 1024),  # walls: no level qualifies
}


@pytest.mark.parametrize("name", list(STREAM_CASES))
def test_row_streaming_matches_vectorized_kernels(name):
    """Periodic lattice levels on the row-streaming kernels (tiles = 5): every
    multi-CTA level of the periodic meshes (down to 2 x 2 blocks, strips
    wrapping around both axes), none of the channel's.  The V-cycle equals
    the six-launch one to rounding (the same row arithmetic; only the coarse
    sums fold in another order), twice (buffers reused), and the solves match
    the oracle with the untiled layout's iteration counts."""
    spec, nstream, tail = STREAM_CASES[name]
    m = BlockTreeMesh(**spec)
    s = EllipticSolver(PoissonOperator(m), multigrid=MultigridOptions(coarse_size=64))
    s0 = EllipticSolver(PoissonOperator(m), multigrid=MultigridOptions(coarse_size=64))
    s.set_tuning(tiles=5, tail_cells=tail)
    s0.set_tuning(tiles=0, tail_cells=tail)
    assert s.streamed_levels() == nstream and s0.streamed_levels() == 0
    rng = np.random.default_rng(6)
    vol = m.cell_volumes()
    for trial in range(2):
        r = rng.standard_normal(m.ncells) * vol
        r -= vol * np.sum(r) / np.sum(vol)
        for precision, tol in (("fp64", 1e-13), ("mixed", 1e-5)):
            z, z0 = s.vcycle(r, precision=precision), s0.vcycle(r, precision=precision)
            assert np.max(np.abs(z - z0)) <= tol * np.max(np.abs(z0)), (precision, trial)
    oo = OOp(block_tree_mesh(**spec), np.ones(m.nfaces))
    rhs = W.gaussian_rhs(m, 8)
    po, _ = osolve(oo, TreeGeometricMultigrid(oo, OMG(coarse_size=64)), rhs, rtol=1e-12)
    for precision, rtol, tol in (("fp64", 1e-12, 1e-10), ("mixed", 1e-10, 1e-9)):
        x, x0 = np.zeros(m.ncells), np.zeros(m.ncells)
        st = solve(x, s, rhs, rtol=rtol, precision=precision)
        st0 = solve(x0, s0, rhs, rtol=rtol, precision=precision)
        assert st.converged and st.cycles == st0.cycles, (precision, st.cycles, st0.cycles)
        assert np.max(np.abs(x - po)) <= tol * np.max(np.abs(po)), precision


def test_row_streaming_on_the_large_levels_only():
    """tiles = 4 on 1024^2: the 1M-cell finest level on the row-streaming
    kernels, the levels of at most 2^19 cells on stencil tiles.  The V-cycle
    equals the six-launch one to rounding, and the solves take the same number
    of iterations to the same solution, in every precision."""
    m = BlockTreeMesh(base_mesh=(1024, 1024), block_size=(16, 16), periodic=(True, True))
    s = EllipticSolver(PoissonOperator(m))
    s0 = EllipticSolver(PoissonOperator(m))
    s.set_tuning(tiles=4, tail_cells=1024)
    s0.set_tuning(tiles=0, tail_cells=1024)
    multi = [n for n in s.level_sizes()[:-1] if n > 1024]
    assert s.streamed_levels() == 1 and s.tiled_levels() == len(multi)
    rng = np.random.default_rng(12)
    r = rng.standard_normal(m.ncells)
    r -= r.mean()
    r *= m.cell_volumes()
    for precision, tol in (("fp64", 1e-13), ("mixed", 1e-5)):
        z, z0 = s.vcycle(r, precision=precision), s0.vcycle(r, precision=precision)
        assert np.max(np.abs(z - z0)) <= tol * np.max(np.abs(z0)), precision
    rhs = r / m.cell_volumes()
    for precision in ("fp64", "mixed", "mixed_ir"):
        x, x0 = np.zeros(m.ncells), np.zeros(m.ncells)
        st = solve(x, s, rhs, rtol=1e-10, precision=precision)
        st0 = solve(x0, s0, rhs, rtol=1e-10, precision=precision)
        assert st.converged and st0.converged and st.cycles == st0.cycles, precision
        assert np.max(np.abs(x - x0)) <= 1e-9 * np.max(np.abs(x0)), precision
