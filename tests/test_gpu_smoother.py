"""The red-black Gauss-Seidel smoother on the B200 against the oracle's
red-black V-cycle (oracle/multigrid.py, `smoother="red_black"`).

Tolerances as for the damped-Jacobi cycle: one FP64 V-cycle to 1e-10
relative, mixed to 1e-4; FP64 solutions to 1e-10 relative after rtol 1e-12
solves, mixed to 1e-9.  The cycle must stay symmetric (red then black before
the coarse correction, black then red after it): <M r1, r2> = <r1, M r2> to
1e-12.
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
from tpagmg._lib import TpaError  # noqa: E402

CASES = {
    # exact two-colouring on every level, all levels beyond the tail
    "taylor_green_128": (W.taylor_green_spec(), None),
    # AMR levels couple cells of one colour; multi-CTA levels and the tail
    "droplet_l2": (W.droplet_spec(levels=2), "droplet"),
    "pruned_varcoef": (dict(block_size=(8, 8), max_level=3,
                            refine=lambda k, o, e: k[0] == 0 or (k[0] < 3 and o[0] < 0.5 and o[1] < 0.5)),
                       "sin"),
    # walls, every level inside the single-CTA tail
    "walls_affine": (dict(base_mesh=(16, 16), block_size=(4, 4), origin=(-1.0, 0.25), extent=(2.0, 1.5),
                          periodic=(False, False)), "cos"),
}


def coefficients(m, kind):
    if kind is None:
        return np.ones(m.nfaces)
    if kind == "droplet":
        return W.droplet_inputs(m)[1]
    if kind == "sin":
        return np.exp(0.4 * np.sin(np.arange(m.nfaces) + 1.0))
    return 3.0 + 0.3 * np.cos(np.arange(m.nfaces))


def build(name, sweeps=2, precision="fp64"):
    spec, kind = CASES[name]
    m = BlockTreeMesh(**spec)
    kappa = coefficients(m, kind)
    s = EllipticSolver(PoissonOperator(m, kappa), preconditioner_options={"precision": precision},
                       multigrid=MultigridOptions(smoother="red_black", pre_sweeps=sweeps, post_sweeps=sweeps))
    oo = OOp(block_tree_mesh(**spec), kappa)
    mg = TreeGeometricMultigrid(oo, OMG(smoother="red_black", pre_sweeps=sweeps, post_sweeps=sweeps))
    return m, s, oo, mg


def residual(m, oo, seed):
    r = np.random.default_rng(seed).standard_normal(m.ncells) * oo.volumes
    return r - oo.volumes * np.sum(r) / np.sum(oo.volumes)


@pytest.mark.parametrize("sweeps", [2, 1, 3])
@pytest.mark.parametrize("name", list(CASES))
def test_red_black_vcycle_matches_oracle(name, sweeps):
    """sweeps 2: the fused cycle (multi-CTA kernels and the coarse tail);
    1 and 3: the plain per-sweep cycle."""
    m, s, oo, mg = build(name, sweeps)
    r = residual(m, oo, 7)
    zo = mg.ldiv(r)
    z = s.vcycle(r, precision="fp64")
    assert np.max(np.abs(z - zo)) <= 1e-10 * np.max(np.abs(zo))
    zf = s.vcycle(r, precision="mixed")
    assert np.max(np.abs(zf - zo)) <= 1e-4 * np.max(np.abs(zo))


@pytest.mark.parametrize("name", list(CASES))
def test_red_black_cycle_is_symmetric(name):
    m, s, oo, mg = build(name)
    r1, r2 = residual(m, oo, 1), residual(m, oo, 2)
    a = float(np.dot(s.vcycle(r1, precision="fp64"), r2))
    b = float(np.dot(r1, s.vcycle(r2, precision="fp64")))
    assert abs(a - b) <= 1e-12 * max(abs(a), abs(b))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", list(CASES))
def test_red_black_solve_matches_oracle(name, precision):
    m, s, oo, mg = build(name, precision=precision)
    rhs = W.taylor_green_rhs(m) if name == "taylor_green_128" else W.gaussian_rhs(m, 11)
    po, so = osolve(oo, mg, rhs, rtol=1e-12)
    x = np.zeros(m.ncells)
    st = solve(x, s, rhs, rtol=1e-12 if precision == "fp64" else 1e-10)
    assert st.converged and so.converged
    tol = 1e-10 if precision == "fp64" else 1e-9
    assert np.max(np.abs(x - po)) <= tol * np.max(np.abs(po))
    # the Jacobi-smoothed solve reaches the same solution in no fewer iterations
    sj = EllipticSolver(PoissonOperator(m, coefficients(m, CASES[name][1])),
                        preconditioner_options={"precision": precision})
    xj = np.zeros(m.ncells)
    stj = solve(xj, sj, rhs, rtol=1e-12 if precision == "fp64" else 1e-10)
    assert stj.converged and st.cycles <= stj.cycles
    assert np.max(np.abs(xj - x)) <= tol * np.max(np.abs(po))


def test_red_black_after_device_refresh(monkeypatch):
    """The device refresh recomputes the half-sweep weights too."""
    spec, _ = CASES["droplet_l2"]
    m = BlockTreeMesh(**spec)
    k1 = np.exp(np.random.default_rng(1).uniform(-2, 2, m.nfaces))
    k2 = np.exp(np.random.default_rng(2).uniform(-2, 2, m.nfaces))
    opts = MultigridOptions(smoother="red_black")
    dev = EllipticSolver(PoissonOperator(m, k1), multigrid=opts)
    host = EllipticSolver(PoissonOperator(m, k1), multigrid=opts)
    r = np.random.default_rng(3).standard_normal(m.ncells) * m.cell_volumes()
    dev.vcycle(r)
    host.vcycle(r)
    dev.refresh(k2)
    assert dev.last_refresh()[0] == "device"
    monkeypatch.setenv("TPAGMG_HOST_REFRESH", "1")
    host.refresh(k2)
    monkeypatch.delenv("TPAGMG_HOST_REFRESH")
    za, zb = dev.vcycle(r, precision="fp64"), host.vcycle(r, precision="fp64")
    assert np.max(np.abs(za - zb)) <= 1e-12 * np.max(np.abs(zb))


def test_merged_batch_rejects_red_black():
    from tpagmg import BatchedSolver
    spec, _ = CASES["walls_affine"]
    m = BlockTreeMesh(**spec)
    s = EllipticSolver(PoissonOperator(m, np.ones(m.nfaces)), multigrid=MultigridOptions(smoother="red_black"))
    with pytest.raises(TpaError) as e:
        BatchedSolver([s])
    assert e.value.code == 5
