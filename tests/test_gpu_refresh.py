"""The coefficient refresh on the device (`_refresh_geometric_multigrid!`,
src/solvers/multigrid/geometric_preconditioner.jl:483-594) against the host
refresh and the CPU oracle.

Tolerances: operator action 1e-14 of |A||x| (the device sums each entry's
contributions in another order); one FP64 V-cycle 1e-12 relative (weights and
the coarse inverse agree to rounding); one mixed V-cycle 1e-6; solutions after
rtol 1e-12 solves 1e-10 relative to the oracle's.
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


def two_level(bs):
    return dict(block_size=(bs, bs), max_level=2,
                refine=lambda k, o, e: k[0] == 0 or (k[0] == 1 and k[1] == 0 and k[2] == 0))


CASES = {
    "two_level_b8": (two_level(8), 8),
    "pruned_b8": (dict(block_size=(8, 8), max_level=3,
                       refine=lambda k, o, e: k[0] == 0 or (k[0] < 3 and o[0] < 0.5 and o[1] < 0.5)), 64),
    "walls_affine": (dict(base_mesh=(16, 16), block_size=(4, 4), origin=(-1.0, 0.25), extent=(2.0, 1.5),
                          periodic=(False, False)), 16),
    "droplet_l2": (W.droplet_spec(levels=2), 64),
    # coarsest matrix of 1025 unknowns: too large for the cluster's shared
    # memory, factored by one CTA in global memory
    "droplet_l2_coarse1024": (W.droplet_spec(levels=2), 1024),
}


def coefficients(m, seed):
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(-2.0, 2.0, m.nfaces))


def solver(m, kappa, coarse):
    s = EllipticSolver(PoissonOperator(m, kappa), multigrid=MultigridOptions(coarse_size=coarse))
    s.set_tuning(structured=0)  # CSR levels: the device refresh applies
    return s


def zero_mean_residual(m, seed):
    vol = m.cell_volumes()
    r = np.random.default_rng(seed).standard_normal(m.ncells) * vol
    return r - vol * np.sum(r) / np.sum(vol)


@pytest.mark.parametrize("case,lu", [(c, "cluster") for c in CASES] + [("pruned_b8", "one_cta"),
                                                                         ("droplet_l2", "one_cta")])
def test_device_refresh_matches_host_refresh(case, lu, monkeypatch):
    spec, coarse = CASES[case]
    m = BlockTreeMesh(**spec)
    k1, k2 = coefficients(m, 1), coefficients(m, 2)
    if lu == "one_cta":
        monkeypatch.setenv("TPAGMG_LU_ONE_CTA", "1")  # read when the refresh is first prepared
    dev = solver(m, k1, coarse)
    host = solver(m, k1, coarse)
    r = zero_mean_residual(m, 3)
    dev.vcycle(r)  # uploads the hierarchy
    host.vcycle(r)
    dev.refresh(k2)
    assert dev.last_refresh()[0] == "device"
    monkeypatch.delenv("TPAGMG_LU_ONE_CTA", raising=False)
    monkeypatch.setenv("TPAGMG_HOST_REFRESH", "1")
    host.refresh(k2)
    monkeypatch.delenv("TPAGMG_HOST_REFRESH")
    assert host.last_refresh()[0] == "host"
    x = np.random.default_rng(5).standard_normal(m.ncells)
    ya, yb = dev.apply(x), host.apply(x)
    scale = np.max(np.abs(yb)) + 1e-300
    assert np.max(np.abs(ya - yb)) <= 1e-13 * scale
    for precision, tol in (("fp64", 1e-12), ("mixed", 1e-6)):
        za, zb = dev.vcycle(r, precision), host.vcycle(r, precision)
        assert np.max(np.abs(za - zb)) <= tol * np.max(np.abs(zb)), precision
    # host queries see the refreshed levels
    for level in range(len(host.level_sizes())):
        wa, wb = dev.level_info(level), host.level_info(level)
        assert wa == wb


@pytest.mark.parametrize("case", ["pruned_b8", "droplet_l2"])
def test_lu_forms_agree_bitwise(case, monkeypatch):
    """The cluster LU and the one-CTA LU apply the same operations to every
    element in the same order, so the refreshed V-cycles agree bit for bit."""
    spec, coarse = CASES[case]
    m = BlockTreeMesh(**spec)
    k1, k2 = coefficients(m, 1), coefficients(m, 2)
    r = zero_mean_residual(m, 3)
    out = []
    for one_cta in (False, True):
        if one_cta:
            monkeypatch.setenv("TPAGMG_LU_ONE_CTA", "1")
        s = solver(m, k1, coarse)
        s.vcycle(r)
        s.refresh(k2)
        assert s.last_refresh()[0] == "device"
        out.append(s.vcycle(r, "fp64"))
    monkeypatch.delenv("TPAGMG_LU_ONE_CTA")
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("case", ["pruned_b8", "droplet_l2"])
def test_device_refresh_solves_match_oracle(case):
    """A chain of device refreshes, then solves at the last coefficients agree
    with the oracle's hierarchy built on them."""
    spec, coarse = CASES[case]
    m = BlockTreeMesh(**spec)
    s = solver(m, coefficients(m, 10), coarse)
    rhs = W.gaussian_rhs(m, 4)
    x = np.zeros(m.ncells)
    solve(x, s, rhs, rtol=1e-12)
    for seed in (11, 12, 13):
        kappa = coefficients(m, seed)
        s.refresh(kappa)
        assert s.last_refresh()[0] == "device"
    oo = OOp(block_tree_mesh(**spec), kappa)
    ref, ost = osolve(oo, TreeGeometricMultigrid(oo, OMG(coarse_size=coarse)), rhs, rtol=1e-12)
    for precision, tol in (("fp64", 1e-10), ("mixed", 1e-9)):
        x = np.zeros(m.ncells)
        st = solve(x, s, rhs, rtol=1e-12 if precision == "fp64" else 1e-10, precision=precision)
        assert st.converged and ost.converged
        assert np.max(np.abs(x - ref)) <= tol * np.max(np.abs(ref)), precision


def test_refresh_with_new_zero_faces_takes_the_host_path():
    """Zeroing coefficients changes the components, so the host rebuilds;
    the solve still matches a freshly built hierarchy."""
    spec, coarse = CASES["pruned_b8"]
    m = BlockTreeMesh(**spec)
    k1 = coefficients(m, 20)
    s = solver(m, k1, coarse)
    rhs = W.gaussian_rhs(m, 6)
    x = np.zeros(m.ncells)
    solve(x, s, rhs, rtol=1e-12)
    k2 = k1.copy()
    k2[::7] = 0.0
    s.refresh(k2)
    assert s.last_refresh()[0] == "host"
    s.refresh(k2 * 3.0)  # same zero set: back on the device
    assert s.last_refresh()[0] == "device"
    fresh = solver(m, k2 * 3.0, coarse)
    a, b = np.zeros(m.ncells), np.zeros(m.ncells)
    solve(a, s, rhs, rtol=1e-12)
    solve(b, fresh, rhs, rtol=1e-12)
    assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(b))


@pytest.mark.parametrize("case", ["pruned_b8", "droplet_l2"])
def test_device_refresh_of_stencil_levels(case, monkeypatch):
    """Variable-coefficient block-structured levels (stencil couplings plus
    exception rows): the device refresh gathers their copies from the refreshed
    operator; the cycle matches the host refresh and solves match the oracle."""
    spec, coarse = CASES[case]
    m = BlockTreeMesh(**spec)
    k1, k2 = coefficients(m, 31), coefficients(m, 32)

    def stencil_solver():
        s = EllipticSolver(PoissonOperator(m, k1), multigrid=MultigridOptions(coarse_size=coarse))
        s.set_tuning(structured=2, tail_cells=64)
        return s

    dev, host = stencil_solver(), stencil_solver()
    assert dev.device_info()["structured_levels"] >= 1
    dev.refresh(k2)
    assert dev.last_refresh()[0] == "device"
    monkeypatch.setenv("TPAGMG_HOST_REFRESH", "1")
    host.refresh(k2)
    monkeypatch.delenv("TPAGMG_HOST_REFRESH")
    assert dev.device_info()["structured_levels"] == host.device_info()["structured_levels"] >= 1
    r = zero_mean_residual(m, 33)
    for precision, tol in (("fp64", 1e-12), ("mixed", 1e-6)):
        za, zb = dev.vcycle(r, precision), host.vcycle(r, precision)
        assert np.max(np.abs(za - zb)) <= tol * np.max(np.abs(zb)), precision
    rhs = W.gaussian_rhs(m, 34)
    oo = OOp(block_tree_mesh(**spec), k2)
    ref, _ = osolve(oo, TreeGeometricMultigrid(oo, OMG(coarse_size=coarse)), rhs, rtol=1e-12)
    x = np.zeros(m.ncells)
    assert solve(x, dev, rhs, rtol=1e-12).converged
    assert np.max(np.abs(x - ref)) <= 1e-10 * np.max(np.abs(ref))


def test_refresh_of_structured_levels_takes_the_host_path():
    """Levels kept as one constant coupling change layout when the
    coefficients vary: refreshed on the host."""
    m = BlockTreeMesh(**W.taylor_green_spec())
    s = EllipticSolver(PoissonOperator(m), multigrid=MultigridOptions(coarse_size=64))
    assert s.device_info()["structured_levels"] >= 1
    s.refresh(np.full(m.nfaces, 2.0))
    assert s.last_refresh()[0] == "host"
