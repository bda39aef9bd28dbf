"""The V-cycle layout autotuner: every candidate layout gives the same V-cycle
(FP64, to 1e-12 relative; they differ in data movement only), the tuner keeps
the fastest measured layout, and solves after tuning still match the oracle."""
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


def droplet():
    spec = W.droplet_spec(levels=2)
    m = BlockTreeMesh(**spec)
    _, kappa, _ = W.droplet_inputs(m)
    return spec, m, kappa


@pytest.mark.parametrize("layout", [dict(tail_cells=512), dict(tail_cells=8192, tail_ctas=4),
                                    dict(structured=0), dict(structured=2), dict(pdl=0), dict(fuse_restrict=1), dict(fuse_restrict=16384),
                                    dict(persistent=1), dict(persistent=1, tail_cells=4096),
                                    dict(tail_cells=1024, tail_ctas=8, structured=2, pdl=0)])
def test_every_layout_gives_the_same_vcycle(layout):
    spec, m, kappa = droplet()
    s = EllipticSolver(PoissonOperator(m, kappa), multigrid=MultigridOptions(coarse_size=64))
    vol = m.cell_volumes()
    r = np.random.default_rng(5).standard_normal(m.ncells) * vol
    r -= vol * r.sum() / vol.sum()
    z0 = s.vcycle(r, precision="fp64")
    s.set_tuning(**layout)
    t = s.tuning()
    for k, v in layout.items():
        assert t[k] == v
    z1 = s.vcycle(r, precision="fp64")
    assert np.max(np.abs(z1 - z0)) <= 1e-12 * np.max(np.abs(z0))


def test_autotune_keeps_the_fastest_layout_and_solves_match_the_oracle():
    spec, m, kappa = droplet()
    s = EllipticSolver(PoissonOperator(m, kappa), multigrid=MultigridOptions(coarse_size=64),
                       preconditioner_options={"precision": "mixed"})
    best, tried = s.autotune(vcycles=5)
    assert len(tried) >= 16 and all(t["ms_per_vcycle"] > 0 for t in tried)
    assert best["ms_per_vcycle"] == min(t["ms_per_vcycle"] for t in tried)
    now = s.tuning()
    for k in ("tail_cells", "tail_ctas", "structured", "vectorized", "pdl", "fuse_restrict", "persistent"):
        assert now[k] == best[k]
    rhs = W.gaussian_rhs(m, 8)
    oo = OOp(block_tree_mesh(**spec), kappa)
    po, so = osolve(oo, TreeGeometricMultigrid(oo, OMG(coarse_size=64)), rhs, rtol=1e-12)
    x = np.zeros(m.ncells)
    assert solve(x, s, rhs, rtol=1e-10).converged
    assert np.max(np.abs(x - po)) <= 1e-9 * np.max(np.abs(po))
    # the layout survives a coefficient refresh
    s.refresh(kappa * 2.0)
    assert s.tuning()["tail_cells"] == best["tail_cells"]


def test_bad_layouts_are_rejected():
    spec, m, kappa = droplet()
    s = EllipticSolver(PoissonOperator(m, kappa))
    with pytest.raises(TpaError):
        s.set_tuning(tail_ctas=9)
    with pytest.raises(ValueError):
        s.set_tuning(tiling=3)  # not a layout field
