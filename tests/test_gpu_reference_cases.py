"""Reference testsets of the solve path run through the C-ABI on the B200
(test/operators/poisson.jl of ronaldremmerswaal/TwoPhaseAMR.jl), beside the
oracle's restatements in test_oracle_golden.py.

Bars are the reference's own: solutions within 1e-6 of the manufactured field
at rtol 1e-8 (:672-720); the strong-form action equal to minus the divergence
of the weighted gradient to atol 2e-11, rtol 2e-13 (:788-818); preconditioned
solutions within 2e-9 of one another at rtol 1e-10 (:833-882).  Solutions are
also held to the oracle's: 1e-10 relative in FP64, 1e-9 mixed.
"""
import numpy as np
import pytest

from oracle import projection as OP
from oracle.krylov import solve as osolve
from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions as OMG, TreeGeometricMultigrid
from oracle.operator import PoissonOperator as OOp
from reference_cases import chain_exact, chain_spec, deep_rhs, deep_spec, harmonic_face_coefficients, two_level_spec

pytestmark = pytest.mark.gpu

from tpagmg import BlockTreeMesh, EllipticSolver, MultigridOptions, PoissonOperator, solve  # noqa: E402
from tpagmg import projection as P  # noqa: E402


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_root_block_vcycle_cg_comparison(precision):
    """:672-720: four levels capped (coarsest the 8x8-cell root level) against
    five uncapped (down to one 4x4 block), four sweeps each way."""
    spec = chain_spec()
    m = BlockTreeMesh(**spec)
    capped = EllipticSolver(PoissonOperator(m), preconditioner_options={"precision": precision},
                            multigrid=MultigridOptions(coarse_size=16, max_levels=4, pre_sweeps=4, post_sweeps=4))
    full = EllipticSolver(PoissonOperator(m), preconditioner_options={"precision": precision},
                          multigrid=MultigridOptions(coarse_size=16, pre_sweeps=4, post_sweeps=4))
    assert len(capped.level_sizes()) == 4 and len(full.level_sizes()) == 5
    assert capped.level_sizes()[-1] == 64 and full.level_sizes()[-1] == 16
    x, y = m.cell_centers()
    exact = chain_exact(x, y)
    vol = m.cell_volumes()
    rhs = full.apply(exact) / vol  # `apply!`: the strong form
    exact = exact - np.dot(vol, exact) / np.sum(vol)
    om = block_tree_mesh(**spec)
    oop = OOp(om)
    po, _ = osolve(oop, TreeGeometricMultigrid(oop, OMG(coarse_size=16, pre_sweeps=4, post_sweeps=4)), rhs,
                   rtol=1e-12)
    out = []
    for s in (capped, full):
        p = np.zeros(m.ncells)
        st = solve(p, s, rhs, rtol=1e-8, max_cycles=100)
        assert st.converged
        assert np.max(np.abs(p - exact)) <= 1e-6
        assert np.max(np.abs(p - po)) <= 1e-6
        out.append(st.cycles)
    assert out[0] > 1 and out[1] <= out[0]


def test_variable_coefficient_operator():
    """:788-818 on the device: tpa_apply / V = -divergence(weighted_gradient)."""
    spec = two_level_spec(4)
    m = BlockTreeMesh(**spec)
    om = block_tree_mesh(**spec)
    cx, cy = m.cell_centers()
    kappa = harmonic_face_coefficients(om, np.where(cx < 0.5, 1.0, 25.0))
    s = EllipticSolver(PoissonOperator(m, kappa))
    p = np.sin(2 * np.pi * cx) * np.cos(2 * np.pi * cy)
    vol = m.cell_volumes()
    applied = s.apply(p) / vol
    div = P.divergence(P.weighted_gradient(p, s), s)
    assert np.allclose(applied, -div, atol=2e-11, rtol=2e-13)
    oop = OOp(om, kappa)
    ref = oop.apply(p) / oop.volumes
    assert np.allclose(applied, ref, atol=2e-11, rtol=2e-13)
    g, gb = OP.weighted_gradient(oop, p)
    assert np.allclose(div, OP.divergence(om, g, gb), atol=2e-11, rtol=2e-13)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_preconditioned_cg_on_a_deep_tree(precision):
    """:833-882: a tree refined to level 4, coarse_size 32, rtol 1e-10.  The
    device solve converges, agrees with the oracle's preconditioned solve to
    2e-9, and takes fewer cycles than the oracle's plain CG at rtol 1e-8 (the
    device implements the preconditioned solve only)."""
    spec = deep_spec()
    m = BlockTreeMesh(**spec)
    x, y = m.cell_centers()
    rhs = deep_rhs(x, y)
    s = EllipticSolver(PoissonOperator(m), coarse_size=32, preconditioner_options={"precision": precision})
    p = np.zeros(m.ncells)
    st = solve(p, s, rhs, rtol=1e-10, max_cycles=100)
    assert st.converged
    om = block_tree_mesh(**spec)
    oop = OOp(om)
    po, ost = osolve(oop, TreeGeometricMultigrid(oop, OMG(coarse_size=32)), rhs, rtol=1e-10, max_cycles=100)
    assert ost.converged
    assert np.max(np.abs(p - po)) < 2e-9
    _, plain = osolve(oop, None, rhs, rtol=1e-8, max_cycles=500, preconditioner=False)
    assert plain.converged and st.cycles < plain.cycles
