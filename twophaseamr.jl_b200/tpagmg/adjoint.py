"""Differentiable pressure solve: `torch.autograd.Function` over the B200 solve
and its hand-written adjoint (the counterpart of a ChainRulesCore `rrule` for
`solve!`, src/solvers/multigrid/elliptic_solver.jl:628-675 of
ronaldremmerswaal/TwoPhaseAMR.jl, which the reference does not provide).

Forward: p = solve!(solver, rhs) with the face coefficients kappa (the solver's
hierarchy is refreshed, `_refresh_geometric_multigrid!`, when kappa changes).
Backward: one adjoint solve with the same operator (it is symmetric) and the
face kernel, giving dJ/d rhs and dJ/d kappa.  No V-cycle iterate of the
forward solve is kept: the gradient is that of the converged solve.

Tensors may live on the host (float64 CPU) or on the solver's GPU (float64
CUDA); device tensors go through the device entry points on torch's current
stream.
"""
from __future__ import annotations

import numpy as np
import torch

from .solver import solve as _solve


def _same_kappa(solver, kappa_np):
    cur = solver.operator.face_coefficient
    return np.shape(cur) == kappa_np.shape and np.array_equal(np.asarray(cur, dtype=np.float64), kappa_np)


class PressureSolve(torch.autograd.Function):
    """p = PressureSolve.apply(rhs, kappa, solver, rtol, atol, max_cycles, precision)."""

    @staticmethod
    def forward(ctx, rhs, kappa, solver, rtol=1e-10, atol=0.0, max_cycles=100, precision=None):
        if rhs.dtype != torch.float64 or kappa.dtype != torch.float64:
            raise TypeError("rhs and kappa must be float64 tensors")
        kappa_np = kappa.detach().cpu().numpy()
        if not _same_kappa(solver, kappa_np):
            solver.refresh(kappa_np)
        opts = dict(rtol=rtol, atol=atol, max_cycles=max_cycles, precision=precision)
        if rhs.is_cuda:
            rhs_c = rhs.detach().contiguous()
            p = torch.zeros_like(rhs_c)
            solver.set_stream(torch.cuda.current_stream(rhs.device).cuda_stream)
            stats = solver.solve_device(rhs_c.data_ptr(), p.data_ptr(), **opts)
        else:
            p_np = np.zeros(rhs.shape[0])
            stats = _solve(p_np, solver, rhs.detach().numpy(), **opts)
            p = torch.from_numpy(p_np)
        if not stats.converged:
            raise RuntimeError(f"pressure solve did not converge ({stats.cycles} cycles)")
        ctx.solver = solver
        ctx.opts = opts
        ctx.kappa_shape = kappa.shape
        ctx.save_for_backward(p)
        return p

    @staticmethod
    def backward(ctx, grad_p):
        (p,) = ctx.saved_tensors
        solver = ctx.solver
        need_rhs, need_kappa = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        if not (need_rhs or need_kappa):
            return (None,) * 7
        if p.is_cuda:
            g = grad_p.contiguous()
            rhs_bar = torch.empty_like(p)
            kappa_bar = torch.empty(ctx.kappa_shape, dtype=torch.float64, device=p.device)
            solver.set_stream(torch.cuda.current_stream(p.device).cuda_stream)
            stats = solver.adjoint_device(p.data_ptr(), g.data_ptr(), rhs_bar.data_ptr(), kappa_bar.data_ptr(),
                                          **ctx.opts)
        else:
            rb, kb, stats = solver.adjoint(p.numpy(), grad_p.detach().cpu().numpy(), **ctx.opts)
            rhs_bar, kappa_bar = torch.from_numpy(rb), torch.from_numpy(kb)
        if not stats.converged:
            raise RuntimeError(f"adjoint solve did not converge ({stats.cycles} cycles)")
        return (rhs_bar if need_rhs else None, kappa_bar if need_kappa else None, None, None, None, None, None)


def pressure_solve(rhs, kappa, solver, *, rtol=1e-10, atol=0.0, max_cycles=100, precision=None):
    """Differentiable `solve!`: returns p with gradients to rhs and kappa."""
    return PressureSolve.apply(rhs, kappa, solver, rtol, atol, max_cycles, precision)
