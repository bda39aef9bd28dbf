"""Solver options, mirroring the reference's keyword constructors.

`MultigridOptions` follows src/solvers/multigrid/options.jl:14-48 and
`LinearSolverOptions` follows src/solvers/linear_options.jl:54-99 (both in
ronaldremmerswaal/TwoPhaseAMR.jl).  The B200 preconditioner is selected with
`preconditioner="gpu_tree_geometric"`; `preconditioner_options={"precision":
"mixed"}` runs the V-cycle in FP32 inside the FP64 conjugate gradients.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

_PRECONDITIONERS = ("auto", "geometric", "tree_geometric", "gpu_tree_geometric")


def _is_int(v):
    return isinstance(v, (int, np.integer)) and not isinstance(v, bool)


@dataclass(frozen=True)
class MultigridOptions:
    """Geometric-multigrid hierarchy and smoothing configuration."""

    coarse_size: int = 64
    pre_sweeps: int = 2
    post_sweeps: int = 2
    max_levels: int = 32
    # not in the reference: "red_black" replaces the damped Jacobi sweeps by
    # red-black Gauss-Seidel half-sweeps (colour (I + J) mod 2 per level)
    smoother: str = "jacobi"

    def __post_init__(self):
        if self.smoother not in ("jacobi", "red_black"):
            raise ValueError("smoother must be 'jacobi' or 'red_black'")
        if not all(_is_int(v) for v in (self.coarse_size, self.pre_sweeps, self.post_sweeps, self.max_levels)):
            raise TypeError("multigrid sizes and sweep counts must be integers")
        if self.coarse_size <= 0:
            raise ValueError("coarse_size must be positive")
        if self.pre_sweeps < 0:
            raise ValueError("pre_sweeps must be nonnegative")
        if self.post_sweeps < 0:
            raise ValueError("post_sweeps must be nonnegative")
        if self.max_levels <= 0:
            raise ValueError("max_levels must be positive")


@dataclass(frozen=True)
class LinearSolverOptions:
    """Algebraic solver choices shared by the pressure solve."""

    krylov: object = None
    krylov_options: dict = field(default_factory=dict)
    preconditioner: object = "auto"
    preconditioner_options: dict = field(default_factory=dict)

    def __post_init__(self):
        if isinstance(self.krylov, str):
            raise ValueError("krylov must be None, a workspace, or a workspace constructor; strings are not supported")
        if isinstance(self.preconditioner, str) and self.preconditioner not in _PRECONDITIONERS:
            raise ValueError("preconditioner must be 'auto', 'geometric', 'tree_geometric' or 'gpu_tree_geometric'")
        if not isinstance(self.krylov_options, dict):
            raise TypeError("krylov_options must be a dict (a named tuple in Julia)")
        if not isinstance(self.preconditioner_options, dict):
            raise TypeError("preconditioner_options must be a dict (a named tuple in Julia)")
        prec = self.preconditioner_options.get("precision", "fp64")
        if prec not in ("fp64", "mixed"):
            raise ValueError("preconditioner_options precision must be 'fp64' or 'mixed'")
