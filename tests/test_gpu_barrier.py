"""The failure path of the bounded grid barrier of the cooperative V-cycle
(csrc/persistent.cuh).

With the poll limit set to 0 (TPAGMG_BARRIER_SPINS, read when the layout is
applied) every barrier that has to wait gives up at its first unsuccessful
poll, records the error and lets the launch run to its end; the solve then
returns TPA_ERR_TIMEOUT instead of hanging, and the same context solves
correctly once the limit is back to its default.  Nothing waits without a
bound, so the test cannot hang the device."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from tpagmg import BlockTreeMesh, EllipticSolver, PoissonOperator, solve  # noqa: E402
from tpagmg import workloads as W  # noqa: E402
from tpagmg._lib import TPA_ERR_TIMEOUT, TpaError  # noqa: E402


def test_barrier_timeout_is_reported_and_the_context_recovers(monkeypatch):
    m = BlockTreeMesh(**W.droplet_spec(levels=2))
    _, kappa, _ = W.droplet_inputs(m)
    s = EllipticSolver(PoissonOperator(m, kappa))
    rhs = W.gaussian_rhs(m, 31)
    ref = np.zeros(m.ncells)
    assert solve(ref, s, rhs, rtol=1e-10).converged  # default layout
    monkeypatch.setenv("TPAGMG_BARRIER_SPINS", "0")
    s.set_tuning(structured=0, persistent=1, tail_ctas=1)
    assert s.tuning()["persistent"] == 1
    x = np.zeros(m.ncells)
    with pytest.raises(TpaError) as e:
        solve(x, s, rhs, rtol=1e-10, max_cycles=5)
    assert e.value.code == TPA_ERR_TIMEOUT
    with pytest.raises(TpaError) as e:
        s.vcycle(rhs * m.cell_volumes(), precision="fp64")
    assert e.value.code == TPA_ERR_TIMEOUT
    monkeypatch.delenv("TPAGMG_BARRIER_SPINS")
    s.set_tuning(structured=0, persistent=1, tail_ctas=1)
    x = np.zeros(m.ncells)
    st = solve(x, s, rhs, rtol=1e-10)
    assert st.converged
    assert np.max(np.abs(x - ref)) <= 1e-9 * np.max(np.abs(ref))
