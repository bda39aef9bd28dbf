"""Red-black colouring and half-sweep weights of every level, from the
library's host set-up, against the oracle's restatement (oracle/multigrid.py:
`red_black_colours`, `red_black_weight`).  The reference has no colouring (it
smooths with damped Jacobi); the colouring is defined as (I + J) mod 2 at each
cell's own level and is compared bit for bit."""
import numpy as np
import pytest

from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions as OMG, TreeGeometricMultigrid
from oracle.operator import PoissonOperator as OOp

from tpagmg import BlockTreeMesh, EllipticSolver, MultigridOptions, PoissonOperator
from tpagmg import workloads as W

SPECS = {
    "taylor_green_128": W.taylor_green_spec(),
    "droplet_l2": W.droplet_spec(levels=2),
    "pruned_b8": dict(block_size=(8, 8), max_level=3,
                      refine=lambda k, o, e: k[0] == 0 or (k[0] < 3 and o[0] < 0.5 and o[1] < 0.5)),
    "walls_affine": dict(base_mesh=(16, 16), block_size=(4, 4), origin=(-1.0, 0.25), extent=(2.0, 1.5),
                         periodic=(False, False)),
    "channel_48x16": dict(base_mesh=(48, 16), block_size=(8, 8), extent=(3.0, 1.0), periodic=(True, False)),
}


@pytest.mark.parametrize("name", list(SPECS))
def test_colours_and_weights_match_oracle(name):
    spec = SPECS[name]
    m = BlockTreeMesh(**spec)
    kappa = np.exp(0.5 * np.sin(np.arange(m.nfaces) * 0.37))
    s = EllipticSolver(PoissonOperator(m, kappa), multigrid=MultigridOptions(smoother="red_black"))
    om = block_tree_mesh(**spec)
    mg = TreeGeometricMultigrid(OOp(om, kappa), OMG(smoother="red_black"))
    sizes = s.level_sizes()
    assert sizes == mg.level_sizes
    for lev, n in enumerate(sizes):
        col, w = s.level_red_black(lev, n)
        ref = mg.levels[lev]
        assert np.array_equal(col, ref.colours.astype(np.uint8))
        assert abs(w - ref.rb_weight) <= 1e-12
        assert 0.0 < w <= 1.0


def test_smoother_option_is_validated():
    with pytest.raises(ValueError):
        MultigridOptions(smoother="gauss_seidel")
    with pytest.raises(ValueError):
        OMG(smoother="sor")
