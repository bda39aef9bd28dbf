"""The projection step around the solve on the B200 against the oracle
(oracle/projection.py) and the reference's balanced-force known answer
(test/two_phase/forces.jl:110-158 of ronaldremmerswaal/TwoPhaseAMR.jl).

Bars: elementwise kernels (conditional fraction, face coefficients, the
divergence with its per-cell face-order sums, the surface-tension jumps) are
bit-exact; products with the AMR face metric K agree to 1e-14 relative (row
sums in another order; bit-exact where K is diagonal); a projection (which
contains a solve to `tolerance`) agrees with the oracle's to 1e-9 relative in
velocity and pressure; a balanced force projects to |u| < 1e-9.
"""
import numpy as np
import pytest

from oracle import projection as OP
from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions as OMG, TreeGeometricMultigrid
from oracle.operator import PoissonOperator as OOp

pytestmark = pytest.mark.gpu

import torch  # noqa: E402

from tpagmg import BlockTreeMesh, EllipticSolver, MultigridOptions, PoissonOperator  # noqa: E402
from tpagmg import projection as P  # noqa: E402
from tpagmg import workloads as W  # noqa: E402
from tpagmg._lib import TpaError  # noqa: E402

CENTER, RADIUS = (0.5, 0.5), 0.2


def spec_of(kind):
    if kind == "uniform":
        return dict(block_size=(8, 8), max_level=2)
    if kind == "two_level":
        return dict(block_size=(8, 8), max_level=2,
                    refine=lambda k, o, e: k[0] == 0 or (k[0] == 1 and k[1] == 0 and k[2] == 0))
    if kind == "walls":
        return dict(base_mesh=(32, 32), block_size=(8, 8), periodic=(False, False), max_level=1,
                    refine=lambda k, o, e: k[0] == 0 and o[0] < 0.5)
    if kind == "band":
        def cut(k, o, e):
            cx, cy = o[0] + e[0] / 2 - CENTER[0], o[1] + e[1] / 2 - CENTER[1]
            near = np.hypot(max(abs(cx) - e[0] / 2, 0.0), max(abs(cy) - e[1] / 2, 0.0))
            far = np.hypot(abs(cx) + e[0] / 2, abs(cy) + e[1] / 2)
            return near <= RADIUS <= far
        return dict(block_size=(8, 8), max_level=2, refine=cut)
    raise KeyError(kind)


def setup(kind, ratio=1000.0):
    spec = spec_of(kind)
    m = BlockTreeMesh(**spec)
    om = block_tree_mesh(**spec)
    raw = W.circle_fractions(m, CENTER, RADIUS)
    return spec, m, om, raw


def bits(a):
    return np.asarray(a, dtype=np.float64).view(np.uint64)


@pytest.mark.parametrize("kind", ["uniform", "two_level", "walls", "band"])
def test_elementwise_kernels_bit_exact(kind):
    spec, m, om, raw = setup(kind)
    _, ocond = OP.conditional_fraction(raw)
    kappa = OP.face_coefficients(om, ocond, (1000.0, 1.0))
    s = EllipticSolver(PoissonOperator(m, kappa))
    phys, cond = P.conditional_fraction(raw, s)
    ophys, ocond = OP.conditional_fraction(raw)
    assert np.array_equal(bits(phys), bits(ophys)) and np.array_equal(bits(cond), bits(ocond))
    k = P.face_coefficients(cond, s, (1000.0, 1.0))
    assert np.array_equal(bits(k), bits(kappa))
    rng = np.random.default_rng(3)
    u = P.FaceVelocity(m, rng.standard_normal(m.nfaces), rng.standard_normal(m.nboundary_faces))
    d = P.divergence(u, s)
    assert np.array_equal(bits(d), bits(OP.divergence(om, u.interior, u.boundary)))


@pytest.mark.parametrize("kind", ["uniform", "two_level", "walls", "band"])
@pytest.mark.parametrize("formulation", ["csf", "cgfm"])
def test_force_and_weighted_gradient_match_oracle(kind, formulation):
    spec, m, om, raw = setup(kind)
    _, cond = OP.conditional_fraction(raw)
    kappa = OP.face_coefficients(om, cond, (1000.0, 1.0))
    s = EllipticSolver(PoissonOperator(m, kappa))
    oop = OOp(om, kappa)
    a = P.surface_tension(cond, s, sigma=1.0, curvature=5.0, formulation=formulation)
    oa, _ = OP.weighted_jump_force(oop, OP.surface_tension_jumps(om, cond, 1.0, 5.0, formulation))
    scale = np.max(np.abs(oa)) + 1e-300
    assert np.max(np.abs(a.interior - oa)) <= 1e-14 * scale
    assert not np.any(a.boundary)
    p = np.random.default_rng(4).standard_normal(m.ncells)
    g = P.weighted_gradient(p, s)
    og, ogb = OP.weighted_gradient(oop, p)
    assert np.max(np.abs(g.interior - og)) <= 1e-14 * np.max(np.abs(og))
    assert np.array_equal(bits(g.boundary), bits(ogb))
    if kind == "uniform":  # diagonal K: every product is a single rounding
        assert np.array_equal(bits(g.interior), bits(og))


@pytest.mark.parametrize("kind", ["two_level", "walls", "band"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_project_matches_oracle(kind, precision):
    spec, m, om, raw = setup(kind)
    rng = np.random.default_rng(5)
    kappa = np.exp(rng.uniform(-2, 2, m.nfaces))
    s = EllipticSolver(PoissonOperator(m, kappa), preconditioner_options={"precision": precision})
    oop = OOp(om, kappa)
    u0 = rng.standard_normal(m.nfaces)
    ub0 = rng.standard_normal(m.nboundary_faces)
    p0 = rng.standard_normal(m.ncells)
    inh = rng.standard_normal(m.ncells)
    for kw in (dict(), dict(inherited_divergence=inh, reference_dt=0.08), dict(prepared=True)):
        u = P.FaceVelocity(m, u0, ub0)
        p = p0.copy()
        st = P.project(u, p, s, 0.05, tolerance=1e-10, **kw)
        ou, oub, opr, phi, ost = OP.project(oop, TreeGeometricMultigrid(oop, OMG()), u0, ub0, p0, 0.05,
                                            tolerance=1e-10, inherited=kw.get("inherited_divergence"),
                                            reference_dt=kw.get("reference_dt"), prepared=kw.get("prepared", False))
        assert st.converged and ost.converged
        assert st.residual_scale == 1 / 0.05 ** 2 and st.compatible == ost.compatible
        assert np.max(np.abs(u.interior - ou)) <= 1e-9 * np.max(np.abs(ou))
        assert np.max(np.abs(u.boundary - oub), initial=0.0) <= 1e-9 * max(np.max(np.abs(oub), initial=0.0), 1.0)
        assert np.max(np.abs(p - opr)) <= 1e-9 * np.max(np.abs(opr))
        if not kw.get("prepared") and m.nboundary_faces:
            # `project!` makes the walls impermeable first
            assert not np.any(u.boundary)
        # the projected velocity is divergence-free to the solve tolerance, up
        # to the volume mean of the incoming divergence (a net boundary inflow
        # no pressure removes) and the retained part dt w (inh - its mean) of
        # an inherited divergence
        vol = m.cell_volumes()
        d0 = P.divergence(P.FaceVelocity(m, u0, ub0 if kw.get("prepared") else None), s)
        target = np.full(m.ncells, np.sum(vol * d0) / np.sum(vol))
        if "inherited_divergence" in kw:
            w = (0.08 - 0.05) / (0.05 * 0.08)
            target += 0.05 * w * (inh - np.sum(vol * inh) / np.sum(vol))
        assert np.max(np.abs(P.divergence(u, s) - target)) * 0.05 <= 1e-8


@pytest.mark.parametrize("kind", ["uniform", "two_level", "band"])
@pytest.mark.parametrize("ratio", [1.0, 1000.0])
@pytest.mark.parametrize("formulation", ["csf", "cgfm"])
def test_balanced_force_device_pipeline(kind, ratio, formulation):
    """test/two_phase/forces.jl:110-158 on the GPU, every field resident:
    fractions -> kappa -> refresh -> force -> u = dt a -> project! -> |u| < 1e-9."""
    spec, m, om, raw = setup(kind)
    s = EllipticSolver(PoissonOperator(m, np.ones(m.nfaces)))
    step = P.TwoPhaseStep(s, (ratio, 1.0), sigma=1.0, curvature=5.0, formulation=formulation)
    frac = torch.from_numpy(raw).cuda()
    step.update_interface(frac)
    _, cond = OP.conditional_fraction(raw)
    okappa = OP.face_coefficients(om, cond, (ratio, 1.0))
    assert np.array_equal(bits(step.kappa.cpu().numpy()), bits(okappa))
    u = step.force() * 0.01
    ub = torch.zeros(max(m.nboundary_faces, 1), dtype=torch.float64, device="cuda")
    p = torch.zeros(m.ncells, dtype=torch.float64, device="cuda")
    st = step.project(u, ub, p, 0.01, tolerance=1e-11)
    assert st.converged and st.compatible
    assert float(u.abs().max()) < 1e-9
    # the pressure is the CGFM / CSF potential up to a constant
    pot = 5.0 * (cond if formulation == "csf" else (cond > 0.5).astype(float))
    pc = p.cpu().numpy()
    vol = m.cell_volumes()
    diff = (pc - np.sum(vol * pc) / np.sum(vol)) - (pot - np.sum(vol * pot) / np.sum(vol))
    assert np.max(np.abs(diff)) < 1e-4


def test_host_and_device_projection_agree_bitwise():
    spec, m, om, raw = setup("walls")
    rng = np.random.default_rng(9)
    kappa = np.exp(rng.uniform(-1, 1, m.nfaces))
    s = EllipticSolver(PoissonOperator(m, kappa))
    u0, ub0, p0 = rng.standard_normal(m.nfaces), rng.standard_normal(m.nboundary_faces), rng.standard_normal(m.ncells)
    u = P.FaceVelocity(m, u0, ub0)
    p = p0.copy()
    P.project(u, p, s, 0.02, tolerance=1e-10, prepared=True)
    ud, ubd, pd = (torch.from_numpy(a.copy()).cuda() for a in (u0, ub0, p0))
    P.project_device(ud, ubd, pd, s, 0.02, tolerance=1e-10, prepared=True)
    assert np.array_equal(bits(ud.cpu().numpy()), bits(u.interior))
    assert np.array_equal(bits(ubd.cpu().numpy()), bits(u.boundary))
    assert np.array_equal(bits(pd.cpu().numpy()), bits(p))


def test_device_refresh_with_new_zero_faces_falls_back_to_the_host():
    spec, m, om, raw = setup("two_level")
    s = EllipticSolver(PoissonOperator(m, np.ones(m.nfaces)))
    s.set_tuning(structured=0)  # CSR levels: the device refresh applies
    k = torch.ones(m.nfaces, dtype=torch.float64, device="cuda") * 2.0
    P.refresh_device(s, k)
    assert s.last_refresh()[0] == "device"
    k[::5] = 0.0
    P.refresh_device(s, k)
    assert s.last_refresh()[0] == "host"
    P.refresh_device(s, k * 3.0)
    assert s.last_refresh()[0] == "device"
    with pytest.raises(TpaError) as e:
        P.refresh_device(s, k * float("nan"))
    assert e.value.code == 1


def test_argument_errors():
    spec, m, om, raw = setup("uniform")
    s = EllipticSolver(PoissonOperator(m, np.ones(m.nfaces)))
    bad = raw.copy()
    bad[3] = 1.5
    with pytest.raises(TpaError) as e:
        P.conditional_fraction(bad, s)
    assert e.value.code == 1
    u = P.FaceVelocity(m)
    p = np.zeros(m.ncells)
    for kw in (dict(dt=0.0), dict(dt=0.1, tolerance=1.0), dict(dt=0.1, reference_dt=0.05)):
        dt = kw.pop("dt")
        with pytest.raises(TpaError) as e:
            P.project(u, p, s, dt, **kw)
        assert e.value.code == 1
    with pytest.raises(TpaError):
        P.face_coefficients(raw, s, (0.0, 1.0))


def test_projection_on_a_split_domain():
    """Zero coefficients on every face crossing x = 0.5 split a walled box into
    two components: the increment solve projects each component's RHS mean,
    the pressure is re-gauged per component (`_accumulate_pressure_increment!`)
    and `compatible` looks at the largest removed component mean."""
    spec = dict(base_mesh=(32, 32), block_size=(8, 8), periodic=(False, False))
    m = BlockTreeMesh(**spec)
    om = block_tree_mesh(**spec)
    cx, _ = m.face_centers()
    cut = (m.face_axis == 1) & (np.abs(cx - 0.5) < 1e-12)
    kappa = np.where(cut, 0.0, 1.0 + 0.5 * np.sin(np.arange(m.nfaces)))
    s = EllipticSolver(PoissonOperator(m, kappa))
    assert s.level_info(0)[2] == 2
    oop = OOp(om, kappa)
    rng = np.random.default_rng(12)
    u0, ub0, p0 = rng.standard_normal(m.nfaces), rng.standard_normal(m.nboundary_faces), rng.standard_normal(m.ncells)
    for prepared, tol in ((False, 1e-10), (True, 1e-10), (True, 1e-3)):
        u = P.FaceVelocity(m, u0, ub0)
        p = p0.copy()
        st = P.project(u, p, s, 0.05, tolerance=tol, prepared=prepared)
        ou, oub, opr, phi, ost = OP.project(oop, TreeGeometricMultigrid(oop, OMG()), u0, ub0, p0, 0.05,
                                            tolerance=tol, prepared=prepared)
        assert st.converged and ost.converged
        assert st.compatible == ost.compatible
        assert np.max(np.abs(u.interior - ou)) <= 1e-9 * np.max(np.abs(ou))
        assert np.max(np.abs(p - opr)) <= 1e-9 * np.max(np.abs(opr))
        # each component's pressure has volume mean zero
        vol = m.cell_volumes()
        for side in (m.cell_centers()[0] < 0.5, m.cell_centers()[0] > 0.5):
            assert abs(np.sum(vol[side] * p[side])) <= 1e-12 * np.sum(vol[side] * np.abs(p[side]))


def test_projection_after_device_refresh_uses_the_new_coefficients():
    """The face kernels' sqrt(kappa) follows a device refresh (copied on the
    device, the faces stay uploaded)."""
    spec, m, om, raw = setup("two_level")
    rng = np.random.default_rng(21)
    k0 = np.exp(rng.uniform(-1, 1, m.nfaces))
    k1 = np.exp(rng.uniform(-1, 1, m.nfaces))
    s = EllipticSolver(PoissonOperator(m, k0))
    s.set_tuning(structured=0)
    p = rng.standard_normal(m.ncells)
    P.weighted_gradient(p, s)  # faces uploaded with k0
    P.refresh_device(s, torch.from_numpy(k1).cuda())
    assert s.last_refresh()[0] == "device"
    g = P.weighted_gradient(p, s)
    og, _ = OP.weighted_gradient(OOp(om, k1), p)
    assert np.max(np.abs(g.interior - og)) <= 1e-14 * np.max(np.abs(og))
    u0 = rng.standard_normal(m.nfaces)
    u = P.FaceVelocity(m, u0)
    pr = np.zeros(m.ncells)
    P.project(u, pr, s, 0.05, tolerance=1e-10)
    oop = OOp(om, k1)
    ou, _, opr, _, _ = OP.project(oop, TreeGeometricMultigrid(oop, OMG()), u0, None, np.zeros(m.ncells), 0.05,
                                  tolerance=1e-10)
    assert np.max(np.abs(u.interior - ou)) <= 1e-9 * np.max(np.abs(ou))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("coefficient", ["one", "harmonic"])
def test_pressure_projection_known_answer(coefficient, precision):
    """test/operators/poisson.jl:1704-1747 ("pressure projection") through
    `tpa_project`: a sinusoidal velocity on the two-level tree of 8x8 blocks,
    kappa = 1 or the harmonic face mean of (x < 1/2 ? 1 : 100), dt 0.1,
    tolerance 1e-11, coarse_size 8."""
    from reference_cases import harmonic_face_coefficients
    from test_oracle_projection import check_projection_known_answer
    spec = spec_of("two_level")
    m = BlockTreeMesh(**spec)
    om = block_tree_mesh(**spec)
    x, y = m.face_centers()
    u0 = np.where(m.face_axis == 1, np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y),
                  np.cos(2 * np.pi * x) * np.sin(2 * np.pi * y))
    if coefficient == "one":
        kappa = np.ones(m.nfaces)
    else:
        cx, _ = om.cell_centers()
        kappa = harmonic_face_coefficients(om, np.where(cx < 0.5, 1.0, 100.0))
    s = EllipticSolver(PoissonOperator(m, kappa), multigrid=MultigridOptions(coarse_size=8),
                       preconditioner_options={"precision": precision})
    u = P.FaceVelocity(m, u0)
    p = np.zeros(m.ncells)
    st = P.project(u, p, s, 0.1, tolerance=1e-11)
    check_projection_known_answer(st, P.divergence(P.FaceVelocity(m, u0), s), P.divergence(u, s), p,
                                  m.cell_volumes())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_incremental_pressure_projection_known_answer(precision):
    """test/operators/poisson.jl:1749-1771: u = -dt G_k p projects to |u| <
    1e-10 and the pressure to |p| < 1e-9 (one periodic 8x8 block, kappa = 1 +
    cos(2 pi x_f) / 4, tolerance 1e-13)."""
    from test_oracle_projection import incremental_case
    m = BlockTreeMesh(block_size=(8, 8))
    kappa, p0 = incremental_case(block_tree_mesh(block_size=(8, 8)))
    s = EllipticSolver(PoissonOperator(m, kappa), multigrid=MultigridOptions(coarse_size=8),
                       preconditioner_options={"precision": precision})
    g = P.weighted_gradient(p0, s)
    u = P.FaceVelocity(m, -0.1 * g.interior)
    p = p0.copy()
    st = P.project(u, p, s, 0.1, tolerance=1e-13, max_cycles=100)
    assert st.converged
    assert np.max(np.abs(u.interior)) < 1e-10
    assert np.max(np.abs(p)) < 1e-9


def test_projection_argument_validation_leaves_the_velocity():
    """test/operators/poisson.jl:1773-1797 through `tpa_project`."""
    m = BlockTreeMesh(block_size=(4, 4))
    s = EllipticSolver(PoissonOperator(m, np.ones(m.nfaces)), multigrid=MultigridOptions(coarse_size=4))
    u = P.FaceVelocity(m, np.ones(m.nfaces))
    original = u.interior.copy()
    with pytest.raises(ValueError):
        P.project(u, np.zeros(m.ncells), s, 0.1, compatibility="invalid")
    for bad in (0.05, np.inf, np.nan):
        with pytest.raises(TpaError) as e:
            P.project(u, np.zeros(m.ncells), s, 0.1, reference_dt=bad)
        assert e.value.code == 1
        assert np.array_equal(u.interior, original)
    for bad in (0.0, -np.finfo(float).eps, 1.0, np.inf, np.nan):
        with pytest.raises(TpaError) as e:
            P.project(u, np.zeros(m.ncells), s, 0.1, tolerance=bad)
        assert e.value.code == 1
        assert np.array_equal(u.interior, original)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mixed_level_no_permeation_projection_known_answer(precision):
    """test/operators/poisson.jl:1799-1823: a walled two-level tree of 4x4
    blocks, u = (0.3 + sin cos, -0.2 + cos sin), dt 0.05, tolerance 1e-10, 80
    cycles: converged, max |div u| <= 1e-8, zero boundary velocity, pressure
    integral <= 2e-11."""
    from test_oracle_projection import no_permeation_case
    spec, om, u0, ub0 = no_permeation_case()
    m = BlockTreeMesh(**spec)
    assert np.array_equal(m.face_axis, om.face_axis) and np.array_equal(m.bface_cell, om.bface_cell)
    s = EllipticSolver(PoissonOperator(m, np.ones(m.nfaces)), multigrid=MultigridOptions(coarse_size=8),
                       preconditioner_options={"precision": precision})
    u = P.FaceVelocity(m, u0, ub0)
    p = np.zeros(m.ncells)
    st = P.project(u, p, s, 0.05, tolerance=1e-10, max_cycles=80)
    assert st.converged
    assert np.max(np.abs(P.divergence(u, s))) <= 1e-8
    assert not np.any(u.boundary)
    assert abs(np.sum(m.cell_volumes() * p)) <= 2e-11
