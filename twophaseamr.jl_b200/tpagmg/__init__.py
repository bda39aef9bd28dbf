"""tpagmg: B200-native drop-in for TwoPhaseAMR.jl's one-velocity pressure solve.

Host-side mirror of the reference's interface for this path (names, argument
meaning and error behaviour as in ronaldremmerswaal/TwoPhaseAMR.jl):

  BlockTreeMesh        src/mesh/topology/mesh.jl:1059-1121
  PoissonOperator      src/operators/elliptic.jl:969-980, two_phase/forces.jl:113-140
  MultigridOptions     src/solvers/multigrid/options.jl:14-48
  LinearSolverOptions  src/solvers/linear_options.jl:54-99
  EllipticSolver       src/solvers/multigrid/elliptic_solver.jl:211-302
  solve (solve!)       src/solvers/multigrid/elliptic_solver.jl:614-675
  LinearSolverStats    src/solvers/multigrid/stats.jl:100-135
  project (project!)   src/navier_stokes/projection.jl:183-260, with divergence!,
                       weighted_gradient!, surface_tension! and FaceVelocity

Every solve runs on the GPU through `libtpagmg.so`; there is no CPU path.
"""
from .mesh import BlockTreeMesh
from .options import LinearSolverOptions, MultigridOptions
from .operator import PoissonOperator, mixture_density, surface_tension_jumps
from .solver import EllipticSolver, LinearSolverStats, solve, solve_batched
from .batch import BatchedSolver
from .projection import FaceVelocity, project, divergence, weighted_gradient, surface_tension

__all__ = ["BlockTreeMesh", "PoissonOperator", "MultigridOptions", "LinearSolverOptions", "EllipticSolver",
           "LinearSolverStats", "solve", "solve_batched", "BatchedSolver", "mixture_density",
           "surface_tension_jumps", "FaceVelocity", "project", "divergence", "weighted_gradient",
           "surface_tension"]
