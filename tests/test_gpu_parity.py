"""Parity of the B200 solver (through the C-ABI) with the CPU oracle.

Tolerances: the operator action agrees to 1e-13 of |A||x|; one FP64 V-cycle to
1e-10 relative (different summation order and a dense coarse inverse in place
of the sparse LU); FP64 solutions to 1e-10 relative after both solve to
rtol <= 1e-12; mixed-precision solutions to 1e-9 relative (the stated target).
"""
import numpy as np
import pytest

from oracle.mesh import block_tree_mesh
from oracle.operator import PoissonOperator as OOp
from oracle.multigrid import MultigridOptions as OMG, TreeGeometricMultigrid
from oracle.krylov import solve as osolve

pytestmark = pytest.mark.gpu

from tpagmg import BlockTreeMesh, EllipticSolver, MultigridOptions, PoissonOperator, solve  # noqa: E402
from tpagmg import workloads as W  # noqa: E402
from tpagmg._lib import TpaError  # noqa: E402


def two_level(bs):
    return dict(block_size=(bs, bs), max_level=2,
                refine=lambda k, o, e: k[0] == 0 or (k[0] == 1 and k[1] == 0 and k[2] == 0))


CASES = {
    "two_level_b4": (two_level(4), 8, None),
    "two_level_b16": (two_level(16), 8, None),
    "pruned_varcoef": (dict(block_size=(8, 8), max_level=3,
                            refine=lambda k, o, e: k[0] == 0 or (k[0] < 3 and o[0] < 0.5 and o[1] < 0.5)),
                       64, lambda m: np.exp(0.4 * np.sin(np.arange(m.nfaces) + 1.0))),
    "walls_affine": (dict(base_mesh=(16, 16), block_size=(4, 4), origin=(-1.0, 0.25), extent=(2.0, 1.5),
                          periodic=(False, False)), 16, lambda m: 3.0 + 0.3 * np.cos(np.arange(m.nfaces))),
    "taylor_green_128": (W.taylor_green_spec(), 64, None),
    "droplet_l2": (W.droplet_spec(levels=2), 64, "droplet"),
}


def build(name):
    spec, coarse, coef = CASES[name]
    m = BlockTreeMesh(**spec)
    o = block_tree_mesh(**spec)
    if coef == "droplet":
        _, kappa, _ = W.droplet_inputs(m)
    elif coef is None:
        kappa = np.ones(m.nfaces)
    else:
        kappa = coef(m)
    s = EllipticSolver(PoissonOperator(m, kappa), multigrid=MultigridOptions(coarse_size=coarse))
    oo = OOp(o, kappa)
    mg = TreeGeometricMultigrid(oo, OMG(coarse_size=coarse))
    return m, s, oo, mg


@pytest.mark.parametrize("name", list(CASES))
def test_apply_matches_oracle(name):
    m, s, oo, mg = build(name)
    x = np.sin(0.7 * (np.arange(m.ncells) + 1.0))
    y = s.apply(x)
    ref = oo.matrix @ x
    scale = abs(oo.matrix) @ np.abs(x)
    assert np.all(np.abs(y - ref) <= 1e-13 * scale + 1e-300)
    # the factorized action of the reference agrees to rounding as well
    assert np.max(np.abs(y - oo.apply(x))) <= 1e-12 * np.max(scale)


@pytest.mark.parametrize("name", list(CASES))
def test_vcycle_matches_oracle(name):
    m, s, oo, mg = build(name)
    rng = np.random.default_rng(7)
    r = rng.standard_normal(m.ncells) * oo.volumes
    r -= oo.volumes * np.sum(r) / np.sum(oo.volumes)
    z = s.vcycle(r, precision="fp64")
    zo = mg.ldiv(r)
    assert np.max(np.abs(z - zo)) <= 1e-10 * np.max(np.abs(zo))
    zf = s.vcycle(r, precision="mixed")
    assert np.max(np.abs(zf - zo)) <= 1e-4 * np.max(np.abs(zo))


@pytest.mark.parametrize("name", list(CASES))
def test_solution_matches_oracle(name):
    m, s, oo, mg = build(name)
    if name == "taylor_green_128":
        rhs = W.taylor_green_rhs(m)
    else:
        rhs = W.gaussian_rhs(m, 11)
    po, so = osolve(oo, mg, rhs, rtol=1e-12)
    assert so.converged
    x = np.zeros(m.ncells)
    st = solve(x, s, rhs, rtol=1e-12)
    assert st.converged
    assert abs(st.cycles - so.cycles) <= 2
    assert np.max(np.abs(x - po)) <= 1e-10 * np.max(np.abs(po))
    xm = np.zeros(m.ncells)
    stm = solve(xm, s, rhs, rtol=1e-10, precision="mixed")
    assert stm.converged
    assert np.max(np.abs(xm - po)) <= 1e-9 * np.max(np.abs(po))


@pytest.mark.parametrize("row", [(4, 2.882e-2, 5.587e-2), (8, 6.749e-3, 1.555e-2), (16, 1.643e-3, 4.049e-3)],
                         ids=["b4", "b8", "b16"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_published_manufactured_errors_on_gpu(row, precision):
    """docs/src/poisson.md:253-257 reproduced by the B200 solve."""
    bs, l2_ref, linf_ref = row
    m = BlockTreeMesh(**two_level(bs))
    s = EllipticSolver(PoissonOperator(m), multigrid=MultigridOptions(coarse_size=8),
                       preconditioner_options={"precision": precision})
    x, y = m.cell_centers()
    exact = np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y)
    p = np.zeros(m.ncells)
    st = solve(p, s, 8 * np.pi ** 2 * exact, rtol=1e-10, max_cycles=60)
    assert st.converged
    v = m.cell_volumes()
    err = np.abs(p - exact)
    assert float(f"{np.sqrt(np.sum(v * err ** 2) / np.sum(v)):.3e}") == l2_ref
    assert float(f"{err.max():.3e}") == linf_ref


def test_balanced_force_cgfm():
    """test/two_phase/forces.jl:110-158: the CGFM RHS L psi is balanced by the
    pressure p = psi + const, also at density ratio 1000 on an adapted tree."""
    m = BlockTreeMesh(**W.droplet_spec(levels=2))
    _, kappa, psi = W.droplet_inputs(m)
    s = EllipticSolver(PoissonOperator(m, kappa))
    rhs = W.droplet_rhs(m, s.apply(psi), noise=0.0)
    for precision in ("fp64", "mixed"):
        p = np.zeros(m.ncells)
        st = solve(p, s, rhs, rtol=1e-12 if precision == "fp64" else 1e-10, precision=precision)
        assert st.converged
        v = m.cell_volumes()
        d = p - psi
        d -= np.sum(v * d) / np.sum(v)
        assert np.max(np.abs(d)) <= 1e-8 * np.max(np.abs(psi))


@pytest.mark.parametrize("name", ["taylor_green_128", "droplet_l2"])
def test_structured_levels_match_csr_levels(name, monkeypatch):
    """The block-structured stencil path (with CSR exception rows at coarse-fine
    edges) gives the same V-cycle as the plain CSR path."""
    monkeypatch.setenv("TPAGMG_STRUCTURED", "all")
    m, s, oo, mg = build(name)
    info = s.device_info()
    assert info["structured_levels"] >= 1 and info["fused_cycle"]
    if name == "droplet_l2":
        assert info["exception_rows"] > 0
    rng = np.random.default_rng(3)
    r = rng.standard_normal(m.ncells) * oo.volumes
    r -= oo.volumes * np.sum(r) / np.sum(oo.volumes)
    z = s.vcycle(r, precision="fp64")
    monkeypatch.setenv("TPAGMG_NO_STRUCTURED", "1")
    spec, coarse, coef = CASES[name]
    s2 = EllipticSolver(PoissonOperator(m, s.operator.face_coefficient), multigrid=MultigridOptions(coarse_size=coarse))
    assert s2.device_info()["structured_levels"] == 0
    z2 = s2.vcycle(r, precision="fp64")
    assert np.max(np.abs(z - z2)) <= 1e-12 * np.max(np.abs(z2))
    assert np.max(np.abs(s.apply(r) - s2.apply(r))) <= 1e-13 * np.max(np.abs(s2.apply(r)))


def test_residual_norms_match_oracle():
    """`_integrated_residual_norms` (cycles.jl:210-221) on the device."""
    import torch
    from oracle.krylov import integrated_norms
    m, s, oo, mg = build("droplet_l2")
    r = np.random.default_rng(9).standard_normal(m.ncells) * oo.volumes
    r[5] = -40 * oo.volumes[5]
    rd = torch.from_numpy(r).cuda()
    l2, linf = s.residual_norms_device(rd.data_ptr())
    ol2, olinf = integrated_norms(r, oo.volumes)
    assert l2 == pytest.approx(ol2, rel=1e-12) and linf == pytest.approx(olinf, rel=1e-15)


def test_solves_are_bitwise_repeatable():
    m, s, oo, mg = build("droplet_l2")
    rhs = W.gaussian_rhs(m, 3)
    a = np.zeros(m.ncells)
    b = np.zeros(m.ncells)
    sa = solve(a, s, rhs)
    sb = solve(b, s, rhs)
    assert np.array_equal(a, b) and sa.cycles == sb.cycles


def test_error_paths():
    m, s, oo, mg = build("two_level_b4")
    x = np.zeros(m.ncells)
    bad = np.ones(m.ncells)
    bad[3] = np.nan
    with pytest.raises(TpaError) as e:
        solve(x, s, bad)
    assert e.value.code == 4
    with pytest.raises(TpaError) as e:
        solve(x, s, np.full(m.ncells, 3.0), compatibility="error")
    assert e.value.code == 1
    st = solve(x, s, np.full(m.ncells, 3.0))
    assert st.converged and abs(st.removed_rhs_mean - 3.0) < 1e-12
    assert np.max(np.abs(x)) <= 1e-12
    st = solve(x, s, W.gaussian_rhs(m, 1), max_cycles=0)
    assert st.cycles == 0 and not st.converged


def test_refresh_matches_rebuild():
    """`_refresh_geometric_multigrid!`: new coefficients on the fixed topology
    give the same solve as a freshly built hierarchy."""
    spec = two_level(8)
    m = BlockTreeMesh(**spec)
    k1 = 1.0 + 0.5 * np.sin(np.arange(m.nfaces))
    k2 = np.exp(0.6 * np.cos(np.arange(m.nfaces)))
    s = EllipticSolver(PoissonOperator(m, k1))
    s.refresh(k2)
    fresh = EllipticSolver(PoissonOperator(m, k2))
    rhs = W.gaussian_rhs(m, 5)
    a = np.zeros(m.ncells)
    b = np.zeros(m.ncells)
    solve(a, s, rhs, rtol=1e-12)
    solve(b, fresh, rhs, rtol=1e-12)
    assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))


@pytest.mark.parametrize("spec", [W.taylor_green_spec(), dict(base_mesh=(128, 128), block_size=(16, 16),
                                                              periodic=(False, False)),
                                  dict(base_mesh=(256, 128), block_size=(16, 16), extent=(2.0, 1.0),
                                       periodic=(True, False))],
                         ids=["periodic_128", "walls_128", "channel_256x128"])
def test_vectorized_levels_match_scalar_stencil(spec, monkeypatch):
    """The vectorized constant-coefficient kernels (4-cell quads, walls and
    periodic edges) give the V-cycle, CG operator and solution of the
    one-thread-per-cell stencil kernels and of the oracle."""
    m = BlockTreeMesh(**spec)
    s = EllipticSolver(PoissonOperator(m), multigrid=MultigridOptions(coarse_size=64))
    assert s.device_info()["structured_levels"] >= 1
    monkeypatch.setenv("TPAGMG_NO_VEC", "1")
    s2 = EllipticSolver(PoissonOperator(m), multigrid=MultigridOptions(coarse_size=64))
    monkeypatch.delenv("TPAGMG_NO_VEC")
    rng = np.random.default_rng(4)
    vol = m.cell_volumes()
    r = rng.standard_normal(m.ncells) * vol
    r -= vol * np.sum(r) / np.sum(vol)
    for precision, tol in (("fp64", 1e-12), ("mixed", 1e-5)):
        z, z2 = s.vcycle(r, precision=precision), s2.vcycle(r, precision=precision)
        assert np.max(np.abs(z - z2)) <= tol * np.max(np.abs(z2))
    rhs = W.gaussian_rhs(m, 5)
    x, x2 = np.zeros(m.ncells), np.zeros(m.ncells)
    st, st2 = solve(x, s, rhs, rtol=1e-12), solve(x2, s2, rhs, rtol=1e-12)
    assert st.converged and abs(st.cycles - st2.cycles) <= 1
    assert np.max(np.abs(x - x2)) <= 1e-10 * np.max(np.abs(x2))
    o = block_tree_mesh(**spec)
    oo = OOp(o, np.ones(m.nfaces))
    po, so = osolve(oo, TreeGeometricMultigrid(oo, OMG(coarse_size=64)), rhs, rtol=1e-12)
    assert np.max(np.abs(x - po)) <= 1e-10 * np.max(np.abs(po))
    xm = np.zeros(m.ncells)
    assert solve(xm, s, rhs, rtol=1e-10, precision="mixed").converged
    assert np.max(np.abs(xm - po)) <= 1e-9 * np.max(np.abs(po))


@pytest.mark.parametrize("name", ["droplet_l2", "taylor_green_128", "walls_affine"])
def test_fused_solve_matches_plain_solve(name, monkeypatch):
    """`solve!` with its set-up and checks fused into two passes gives the
    statistics and solution of the kernel-by-kernel path."""
    m, s, oo, mg = build(name)
    rhs = W.gaussian_rhs(m, 13)
    x0 = np.sin(np.arange(m.ncells) * 0.3)
    monkeypatch.setenv("TPAGMG_PLAIN_SOLVE", "1")
    xp = x0.copy()
    sp = solve(xp, s, rhs, rtol=1e-11)
    sp = dict(vars(sp))
    monkeypatch.delenv("TPAGMG_PLAIN_SOLVE")
    for precision in ("fp64", "mixed"):
        xf = x0.copy()
        sf = solve(xf, s, rhs, rtol=1e-11, precision=precision)
        assert sf.converged and sp["converged"]
        assert abs(sf.cycles - sp["cycles"]) <= (1 if precision == "fp64" else 2)
        assert sf.initial_linf == pytest.approx(sp["initial_linf"], rel=1e-12)
        assert sf.initial_l2 == pytest.approx(sp["initial_l2"], rel=1e-12)
        assert sf.removed_rhs_mean == pytest.approx(sp["removed_rhs_mean"], rel=1e-12, abs=1e-300)
        assert np.max(np.abs(xf - xp)) <= 1e-9 * np.max(np.abs(xp))
