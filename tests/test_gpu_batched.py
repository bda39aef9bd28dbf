"""Batched uneven solves (256 independent two-phase problems of tree depth
2..6) through `tpa_solve_batched`: every batched solution is bitwise the one
its own `solve!` gives, the small problems match the oracle, and a failing
problem is reported without stopping the others.

Tolerances: batched vs single solve bit-exact (same context, deterministic
kernels); mixed precision vs the FP64 oracle 1e-9 relative.
"""
import numpy as np
import pytest

from oracle.mesh import block_tree_mesh
from oracle.operator import PoissonOperator as OOp
from oracle.multigrid import MultigridOptions as OMG, TreeGeometricMultigrid
from oracle.krylov import solve as osolve

pytestmark = pytest.mark.gpu

from tpagmg import BlockTreeMesh, EllipticSolver, PoissonOperator, solve, solve_batched  # noqa: E402
from tpagmg import workloads as W  # noqa: E402
from tpagmg._lib import TpaError  # noqa: E402


def make(problems, precision="mixed"):
    out = []
    for p in problems:
        m = BlockTreeMesh(**W.batch_spec(p))
        kappa, rhs = W.batch_inputs(m, p)
        s = EllipticSolver(PoissonOperator(m, kappa), preconditioner_options={"precision": precision})
        out.append((p, m, kappa, rhs, s))
    return out


def small(count):
    return [p for p in W.batch_problems() if p["depth"] <= 3][:count]


def test_batched_equals_single_solves_bitwise():
    probs = make(small(6) + [p for p in W.batch_problems() if p["depth"] == 5][:2])
    xs = [np.zeros(m.ncells) for _, m, *_ in probs]
    stats = solve_batched(xs, [s for *_, s in probs], [r for _, _, _, r, _ in probs], rtol=1e-10, workers=4)
    for (p, m, kappa, rhs, s), x, st in zip(probs, xs, stats):
        assert st.converged
        y = np.zeros(m.ncells)
        st1 = solve(y, s, rhs, rtol=1e-10)
        assert st1.cycles == st.cycles
        assert np.array_equal(x, y)


def test_batched_small_problems_match_oracle():
    probs = make(small(3))
    xs = [np.zeros(m.ncells) for _, m, *_ in probs]
    solve_batched(xs, [s for *_, s in probs], [r for _, _, _, r, _ in probs], rtol=1e-10)
    for (p, m, kappa, rhs, s), x in zip(probs, xs):
        oo = OOp(block_tree_mesh(**W.batch_spec(p)), kappa)
        po, so = osolve(oo, TreeGeometricMultigrid(oo, OMG()), rhs, rtol=1e-12)
        assert so.converged
        assert np.max(np.abs(x - po)) <= 1e-9 * np.max(np.abs(po))


def test_batched_reports_failed_problem_and_solves_the_rest():
    probs = make(small(4))
    xs = [np.zeros(m.ncells) for _, m, *_ in probs]
    rhs = [r.copy() for _, _, _, r, _ in probs]
    rhs[2][5] = np.nan
    with pytest.raises(TpaError, match="problem 2"):
        solve_batched(xs, [s for *_, s in probs], rhs, rtol=1e-10)
    for k in (0, 1, 3):
        assert np.any(xs[k] != 0)


def test_batched_rejects_shared_solver():
    probs = make(small(1))
    _, m, _, rhs, s = probs[0]
    with pytest.raises(ValueError):
        solve_batched([np.zeros(m.ncells), np.zeros(m.ncells)], [s, s], [rhs, rhs])


# ---- merged batch (one launch per V-cycle phase for every problem) ---------------

from tpagmg import BatchedSolver  # noqa: E402


def test_merged_batch_matches_single_solves():
    """FP64: each merged-batch solution agrees with its own context's solve to
    1e-10 relative (both to rtol 1e-12; the smoother weights are folded into
    per-row arrays, so the arithmetic differs at rounding level), with the
    same iteration counts within one; mixed precision to 1e-9."""
    probs = make(small(5) + [p for p in W.batch_problems() if p["depth"] >= 5][:3], precision="fp64")
    bs = BatchedSolver([s for *_, s in probs])
    assert bs.count == len(probs) and bs.levels == max(len(s.level_sizes()) for *_, s in probs)
    rhs = bs.concat([r for _, _, _, r, _ in probs])
    for precision, tol in (("fp64", 1e-10), ("mixed", 1e-9)):
        x = np.zeros(bs.ncells)
        st = bs.solve(x, rhs, rtol=1e-12, precision=precision)
        assert all(s["converged"] for s in st)
        for (p, m, kappa, r, s), xk, sk in zip(probs, bs.split(x), st):
            y = np.zeros(m.ncells)
            s1 = solve(y, s, r, rtol=1e-12, precision=precision)
            assert abs(s1.cycles - sk["cycles"]) <= 1
            assert np.max(np.abs(xk - y)) <= tol * np.max(np.abs(y))


def test_merged_batch_small_problems_match_oracle():
    probs = make(small(3))
    bs = BatchedSolver([s for *_, s in probs])
    x = np.zeros(bs.ncells)
    bs.solve(x, bs.concat([r for _, _, _, r, _ in probs]), rtol=1e-10)
    for (p, m, kappa, rhs, s), xk in zip(probs, bs.split(x)):
        oo = OOp(block_tree_mesh(**W.batch_spec(p)), kappa)
        po, so = osolve(oo, TreeGeometricMultigrid(oo, OMG()), rhs, rtol=1e-12)
        assert np.max(np.abs(xk - po)) <= 1e-9 * np.max(np.abs(po))


def test_merged_batch_device_arrays_and_repeatability():
    import torch
    probs = make(small(4) + [p for p in W.batch_problems() if p["depth"] == 4][:2])
    bs = BatchedSolver([s for *_, s in probs])
    rhs = torch.from_numpy(bs.concat([r for _, _, _, r, _ in probs])).cuda()
    x1 = torch.zeros(bs.ncells, dtype=torch.float64, device="cuda")
    x2 = torch.zeros_like(x1)
    torch.cuda.synchronize()
    bs.solve_device(rhs.data_ptr(), x1.data_ptr(), rtol=1e-10)
    bs.solve_device(rhs.data_ptr(), x2.data_ptr(), rtol=1e-10)
    torch.cuda.synchronize()
    assert torch.equal(x1, x2)
    xh = np.zeros(bs.ncells)
    bs.solve(xh, rhs.cpu().numpy(), rtol=1e-10)
    assert np.array_equal(xh, x1.cpu().numpy())


def test_merged_batch_compatibility_error_marks_one_problem():
    probs = make(small(3))
    bs = BatchedSolver([s for *_, s in probs])
    rhs = [r.copy() for _, _, _, r, _ in probs]
    rhs[1] = rhs[1] + 1.0  # nonzero volume mean
    x = np.zeros(bs.ncells)
    with pytest.raises(TpaError, match="problem 1"):
        bs.solve(x, bs.concat(rhs), rtol=1e-10, compatibility="error")
    parts = bs.split(x)
    assert np.any(parts[0] != 0) and np.any(parts[2] != 0)
    assert not np.any(parts[1] != 0)


def test_merged_batch_after_device_refresh():
    """A context refreshed on the device leaves its host levels stale; the
    merged batch built from it recomputes them first and solves the refreshed
    problem."""
    from tpagmg import BatchedSolver
    probs = make(small(3), precision="fp64")
    p, m, kappa, rhs, s = probs[0]
    s.set_tuning(structured=0)
    k2 = kappa * np.exp(0.3 * np.sin(np.arange(m.nfaces)))
    s.refresh(k2)
    assert s.last_refresh()[0] == "device"
    bs = BatchedSolver([q[-1] for q in probs])
    x = np.zeros(bs.ncells)
    st = bs.solve(x, bs.concat([q[3] for q in probs]), rtol=1e-12, precision="fp64")
    assert all(t["converged"] for t in st)
    oo = OOp(block_tree_mesh(**W.batch_spec(p)), k2)
    ref, _ = osolve(oo, TreeGeometricMultigrid(oo, OMG()), rhs, rtol=1e-12)
    x0 = bs.split(x)[0]
    assert np.max(np.abs(x0 - ref)) <= 1e-10 * np.max(np.abs(ref))


def test_merged_batch_host_driven_loop_matches_graph(monkeypatch):
    """TPAGMG_NO_GRAPH (kernel-by-kernel Krylov loop, condition read on the host;
    the profiling mode) runs the same kernels in the same order as the graph's
    WHILE loop: bit-identical solutions and iteration counts."""
    probs = make(small(4) + [p for p in W.batch_problems() if p["depth"] == 4][:2])
    bs = BatchedSolver([s for *_, s in probs])
    rhs = bs.concat([r for _, _, _, r, _ in probs])
    x1 = np.zeros(bs.ncells)
    st1 = bs.solve(x1, rhs, rtol=1e-10)
    monkeypatch.setenv("TPAGMG_NO_GRAPH", "1")
    x2 = np.zeros(bs.ncells)
    st2 = bs.solve(x2, rhs, rtol=1e-10)
    monkeypatch.delenv("TPAGMG_NO_GRAPH")
    assert [s["cycles"] for s in st1] == [s["cycles"] for s in st2]
    assert np.array_equal(x1, x2)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_single_solve_host_driven_loop_matches_graph(precision, monkeypatch):
    """The same for one solve (graph WHILE loop against kernel-by-kernel)."""
    p = [q for q in W.batch_problems() if q["depth"] == 4][0]
    m = BlockTreeMesh(**W.batch_spec(p))
    kappa, rhs = W.batch_inputs(m, p)
    s = EllipticSolver(PoissonOperator(m, kappa), preconditioner_options={"precision": precision})
    x1 = np.zeros(m.ncells)
    st1 = solve(x1, s, rhs, rtol=1e-10)
    monkeypatch.setenv("TPAGMG_NO_GRAPH", "1")
    x2 = np.zeros(m.ncells)
    st2 = solve(x2, s, rhs, rtol=1e-10)
    monkeypatch.delenv("TPAGMG_NO_GRAPH")
    assert st1.converged and st1.cycles == st2.cycles
    assert np.array_equal(x1, x2)
