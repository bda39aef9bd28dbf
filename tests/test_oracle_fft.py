"""The FFT solve of the uniform periodic pressure system (oracle/fft_poisson.py)
against the assembled oracle: the same operator to rounding, and the same
solution as the oracle's multigrid-preconditioned CG solved to rtol 1e-12.
It is the checker of the 2048^2 GPU solve, where the assembled oracle's set-up
takes too long."""
import numpy as np

from oracle import fft_poisson as F
from oracle.krylov import solve
from oracle.mesh import block_tree_mesh
from oracle.multigrid import MultigridOptions, TreeGeometricMultigrid
from oracle.operator import PoissonOperator
from tpagmg import workloads as W


def test_fft_oracle_matches_assembled_oracle():
    for base, extent in (((128, 128), (1.0, 1.0)), ((128, 64), (2.0, 1.0))):
        spec = dict(base_mesh=base, block_size=(16, 16), extent=extent, periodic=(True, True))
        mesh = block_tree_mesh(**spec)
        op = PoissonOperator(mesh)
        x = np.sin(0.37 * np.arange(mesh.ncells))
        ref = op.apply(x)
        assert np.max(np.abs(F.apply(x, base, (16, 16), extent) - ref)) <= 1e-13 * np.max(np.abs(ref))
        rhs = W.gaussian_rhs(mesh, 303)
        p, st = solve(op, TreeGeometricMultigrid(op, MultigridOptions()), rhs, rtol=1e-12)
        xf = F.solve(rhs, base, (16, 16), extent)
        assert st.converged
        assert np.max(np.abs(xf - p)) <= 1e-10 * np.max(np.abs(xf))
        assert np.allclose(F.from_grid(F.to_grid(x, base, (16, 16)), base, (16, 16)), x, rtol=0, atol=0)
