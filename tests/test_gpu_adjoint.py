"""Adjoint of the pressure solve on the B200 (through the C-ABI and the torch
autograd wrapper): the face kernel against the oracle's formula, the gradients
against the oracle's adjoint (its own CPU solve of the adjoint system), and
against central finite differences (step 1e-6) of the GPU solve along 32
seeded random directions of the right-hand side and of the face coefficients
1/rho, in FP64 and in mixed precision.

Tolerances: face kernel 1e-13 of the largest entry (same formula, different
summation order); gradients vs the oracle 1e-9 relative (both adjoint solves
to rtol 1e-12); finite differences 1e-6 relative per direction plus the
floor of the difference quotient (rounding of J, 64 eps |J| / h, and the two
solves' own error, target * |dJ/drhs|_1 / h each), and over the 32
directions as a vector 1e-6 relative plus the same floors taken as a vector.
The finite-difference tests run on the droplet tree of depth 2 and on the
benchmark's droplet of depth 4 (110,080 cells).
"""
import numpy as np
import pytest

from oracle.adjoint import adjoint as oadjoint, face_gradient as oface_gradient, loss, loss_cotangent, loss_mask
from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions as OMG, TreeGeometricMultigrid
from oracle.operator import PoissonOperator as OOp

pytestmark = pytest.mark.gpu

from tpagmg import BlockTreeMesh, EllipticSolver, MultigridOptions, PoissonOperator, solve  # noqa: E402
from tpagmg import workloads as W  # noqa: E402

H = 1e-6
EPS = np.finfo(np.float64).eps


def two_level_varcoef():
    spec = dict(block_size=(4, 4), max_level=2,
                refine=lambda k, o, e: k[0] == 0 or (k[0] == 1 and k[1] == 0 and k[2] == 0))
    m = BlockTreeMesh(**spec)
    kappa = np.exp(0.5 * np.sin(1.7 * np.arange(m.nfaces) + 0.3))
    return spec, m, kappa, 8


def droplet(levels=2):
    spec = W.droplet_spec(levels=levels)
    m = BlockTreeMesh(**spec)
    _, kappa, _ = W.droplet_inputs(m)
    return spec, m, kappa, 64


def droplet4():
    return droplet(levels=4)


FD_CASES = pytest.mark.parametrize("case", [droplet, droplet4], ids=["droplet_l2", "droplet_l4"])


def setup(case, precision="fp64"):
    spec, m, kappa, coarse = case()
    s = EllipticSolver(PoissonOperator(m, kappa), multigrid=MultigridOptions(coarse_size=coarse),
                       preconditioner_options={"precision": precision})
    return spec, m, kappa, coarse, s


def c5_loss(m, seed=505):
    """J = 1/2 ||p - p_t||^2 over finest cells within 0.2 of the droplet centre."""
    vol = m.cell_volumes()
    mask = loss_mask(m.cell_centers(), center=(0.5, 0.6), radius=0.2, volumes=vol, finest_volume=vol.min())
    target = W.rng(seed).standard_normal(m.ncells)
    return mask, target


@pytest.mark.parametrize("case", [two_level_varcoef, droplet], ids=["two_level_varcoef", "droplet_l2"])
def test_face_kernel_matches_oracle(case):
    spec, m, kappa, coarse, s = setup(case)
    oo = OOp(block_tree_mesh(**spec), kappa)
    rng = np.random.default_rng(3)
    p, lam = rng.standard_normal(m.ncells), rng.standard_normal(m.ncells)
    g = s.face_coefficient_gradient(p, lam)
    go = oface_gradient(oo, p, lam)
    assert np.max(np.abs(g - go)) <= 1e-13 * np.max(np.abs(go))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", [two_level_varcoef, droplet], ids=["two_level_varcoef", "droplet_l2"])
def test_adjoint_matches_oracle_adjoint(case, precision):
    spec, m, kappa, coarse, s = setup(case, precision)
    oo = OOp(block_tree_mesh(**spec), kappa)
    mg = TreeGeometricMultigrid(oo, OMG(coarse_size=coarse))
    rhs = W.gaussian_rhs(m, 17)
    p = np.zeros(m.ncells)
    assert solve(p, s, rhs, rtol=1e-12).converged
    mask, target = c5_loss(m)
    pbar = loss_cotangent(p, target, mask)
    rb, kb, st = s.adjoint(p, pbar, rtol=1e-12)
    assert st.converged
    rbo, kbo, _ = oadjoint(oo, p, pbar, mg, rtol=1e-12)
    assert np.max(np.abs(rb - rbo)) <= 1e-9 * np.max(np.abs(rbo))
    assert np.max(np.abs(kb - kbo)) <= 1e-9 * np.max(np.abs(kbo))


def _J(s, m, rhs, target, mask, precision):
    """Loss of a cold-started solve to rtol 1e-13 and the solve's strong
    residual target."""
    p = np.zeros(m.ncells)
    st = solve(p, s, rhs, rtol=1e-13, precision=precision)
    assert st.converged
    return loss(p, target, mask), p, st.target_linf


def fd_floor(J0, h, targets, rhs_bar):
    """Error floor of a central difference of J: rounding of J, plus the solve
    error, |dJ| <= lam' dr <= target * sum_i |lam_i| V_i = target * |rhs_bar|_1
    for each of the two solves."""
    return 64 * EPS * max(J0, 1.0) / h + sum(targets) * np.sum(np.abs(rhs_bar)) / (2 * h)


@FD_CASES
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rhs_gradient_matches_finite_differences_32_directions(precision, case):
    spec, m, kappa, coarse, s = setup(case, precision)
    rhs = W.droplet_rhs(m, s.apply(W.droplet_inputs(m)[2]))
    mask, target = c5_loss(m)
    J0, p, _ = _J(s, m, rhs, target, mask, precision)
    rb, _, st = s.adjoint(p, loss_cotangent(p, target, mask), rtol=1e-13)
    assert st.converged
    rng = W.rng(5050)
    worst, fds, ads, floors = 0.0, [], [], []
    for _ in range(32):
        d = rng.standard_normal(m.ncells)
        jp, _, tp = _J(s, m, rhs + H * d, target, mask, precision)
        jm, _, tm = _J(s, m, rhs - H * d, target, mask, precision)
        fd = (jp - jm) / (2 * H)
        err = abs(fd - rb @ d)
        floors.append(fd_floor(J0, H, (tp, tm), rb))
        assert err <= 1e-6 * abs(fd) + floors[-1], (fd, rb @ d)
        worst = max(worst, err / abs(fd))
        fds.append(fd)
        ads.append(rb @ d)
    vec = np.linalg.norm(np.subtract(fds, ads)) / np.linalg.norm(fds)
    vec_floor = np.linalg.norm(floors) / np.linalg.norm(fds)
    assert vec <= 1e-6 + vec_floor
    print(f"rhs gradient, {precision}, {m.ncells} cells: worst relative FD mismatch {worst:.2e}, "
          f"over 32 directions {vec:.2e} (floor {vec_floor:.2e})")


@FD_CASES
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_kappa_gradient_matches_finite_differences_32_directions(precision, case):
    spec, m, kappa, coarse, s = setup(case, precision)
    rhs = W.droplet_rhs(m, s.apply(W.droplet_inputs(m)[2]))
    mask, target = c5_loss(m)
    J0, p, _ = _J(s, m, rhs, target, mask, precision)
    rb, kb, st = s.adjoint(p, loss_cotangent(p, target, mask), rtol=1e-13)
    assert st.converged
    rng = W.rng(5051)
    worst, fds, ads, floors = 0.0, [], [], []
    for _ in range(32):
        d = rng.standard_normal(m.nfaces) * kappa
        s.refresh(kappa + H * d)
        jp, _, tp = _J(s, m, rhs, target, mask, precision)
        s.refresh(kappa - H * d)
        jm, _, tm = _J(s, m, rhs, target, mask, precision)
        fd = (jp - jm) / (2 * H)
        err = abs(fd - kb @ d)
        floors.append(fd_floor(J0, H, (tp, tm), rb))
        assert err <= 1e-6 * abs(fd) + floors[-1], (fd, kb @ d)
        worst = max(worst, err / abs(fd))
        fds.append(fd)
        ads.append(kb @ d)
    s.refresh(kappa)
    vec = np.linalg.norm(np.subtract(fds, ads)) / np.linalg.norm(fds)
    vec_floor = np.linalg.norm(floors) / np.linalg.norm(fds)
    assert vec <= 1e-6 + vec_floor
    print(f"kappa gradient, {precision}, {m.ncells} cells: worst relative FD mismatch {worst:.2e}, "
          f"over 32 directions {vec:.2e} (floor {vec_floor:.2e})")


@pytest.mark.parametrize("device", ["cuda", "cpu"])
def test_torch_autograd_matches_adjoint(device):
    import torch
    from tpagmg.adjoint import pressure_solve

    spec, m, kappa, coarse, s = setup(droplet, "mixed")
    rhs_np = W.gaussian_rhs(m, 23)
    mask, target = c5_loss(m)
    rhs = torch.tensor(rhs_np, dtype=torch.float64, device=device, requires_grad=True)
    kap = torch.tensor(kappa, dtype=torch.float64, device=device, requires_grad=True)
    t = torch.tensor(target, dtype=torch.float64, device=device)
    msk = torch.tensor(mask, device=device)
    p = pressure_solve(rhs, kap, s, rtol=1e-12)
    J = 0.5 * torch.sum(torch.where(msk, p - t, torch.zeros_like(p)) ** 2)
    J.backward()
    p_np = p.detach().cpu().numpy()
    rb, kb, _ = s.adjoint(p_np, loss_cotangent(p_np, target, mask), rtol=1e-12)
    np.testing.assert_allclose(rhs.grad.cpu().numpy(), rb, rtol=0, atol=1e-9 * np.max(np.abs(rb)))
    np.testing.assert_allclose(kap.grad.cpu().numpy(), kb, rtol=0, atol=1e-9 * np.max(np.abs(kb)))
    # a changed kappa refreshes the hierarchy and changes the solution
    p2 = pressure_solve(rhs.detach(), (kap * 1.5).detach(), s, rtol=1e-12)
    assert torch.max(torch.abs(p2 - p.detach() / 1.5)) <= 1e-8 * torch.max(torch.abs(p))
    s.refresh(kappa)


def test_adjoint_error_paths():
    spec, m, kappa, coarse, s = setup(two_level_varcoef)
    from tpagmg._lib import TpaError
    with pytest.raises(ValueError):
        s.adjoint(np.zeros(3), np.zeros(3))
    bad = np.zeros(m.ncells)
    bad[0] = np.nan
    with pytest.raises(TpaError):
        s.adjoint(np.zeros(m.ncells), bad)
