"""CPU checks of the batched uneven-solve workload: the seeded problem list
(tree depth U{2..6}, radius U[0.05, 0.3], centre U[0.3, 0.7]^2, density ratio
from {10, 100, 1000}) and bit-exact host set-up of batch problems against the
oracle.  No device computation runs here."""
import numpy as np
import pytest

from oracle.mesh import block_tree_mesh
from oracle.operator import PoissonOperator as OOp
from oracle.multigrid import MultigridOptions as OMG, TreeGeometricMultigrid

from tpagmg import BlockTreeMesh, EllipticSolver, PoissonOperator, solve_batched
from tpagmg import workloads as W


def test_problem_list_is_seeded_and_covers_the_ranges():
    a, b = W.batch_problems(), W.batch_problems()
    assert a == b and len(a) == 256
    assert {p["depth"] for p in a} == {2, 3, 4, 5, 6}
    assert {p["ratio"] for p in a} == {10.0, 100.0, 1000.0}
    assert all(0.05 <= p["radius"] <= 0.3 for p in a)
    assert all(0.3 <= c <= 0.7 for p in a for c in p["center"])
    assert len({p["rhs_seed"] for p in a}) == 256


@pytest.mark.parametrize("k", [0, 1])
def test_batch_problem_host_setup_bit_exact(k):
    p = [q for q in W.batch_problems() if q["depth"] == 2][k]
    spec = W.batch_spec(p)
    m, o = BlockTreeMesh(**spec), block_tree_mesh(**spec)
    assert np.array_equal(m.keys, np.array(o.keys))
    assert np.array_equal(m.face_minus, o.face_minus) and np.array_equal(m.face_plus, o.face_plus)
    kappa, rhs = W.batch_inputs(m, p)
    assert abs(np.dot(rhs, m.cell_volumes())) <= 1e-12 * np.sum(np.abs(rhs) * m.cell_volumes())
    assert kappa.min() == pytest.approx(1.0 / p["ratio"]) and kappa.max() == pytest.approx(1.0)
    s = EllipticSolver(PoissonOperator(m, kappa))
    mg = TreeGeometricMultigrid(OOp(o, kappa), OMG())
    assert s.level_sizes() == mg.level_sizes
    assert s.level_sizes()[-1] == 256
    for lev in range(len(mg.levels) - 1):
        assert np.array_equal(s.level_owners(lev), mg.owners[lev])


def test_batched_argument_checks_need_no_device():
    p = [q for q in W.batch_problems() if q["depth"] == 2][0]
    m = BlockTreeMesh(**W.batch_spec(p))
    kappa, rhs = W.batch_inputs(m, p)
    s = EllipticSolver(PoissonOperator(m, kappa))
    with pytest.raises(ValueError):
        solve_batched([np.zeros(m.ncells)], [s, s], [rhs, rhs])
    with pytest.raises(ValueError):
        solve_batched([np.zeros(m.ncells), np.zeros(m.ncells)], [s, s], [rhs, rhs])
    with pytest.raises(ValueError):
        solve_batched([np.zeros(3)], [s], [rhs])


def test_merged_batch_fails_loudly_without_a_device():
    from tpagmg import BatchedSolver
    from tpagmg._lib import TpaError
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = [q for q in W.batch_problems() if q["depth"] == 2][0]
    m = BlockTreeMesh(**W.batch_spec(p))
    kappa, rhs = W.batch_inputs(m, p)
    s = EllipticSolver(PoissonOperator(m, kappa))
    with pytest.raises(TpaError, match="CUDA device"):
        BatchedSolver([s])
