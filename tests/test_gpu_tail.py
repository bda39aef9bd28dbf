"""The coarse tail staged in shared memory (csrc/tail_smem.cuh, on request:
TPAGMG_TAIL_SMEM) against the default tail that reads its levels from global
memory.  Both run the same phase code
on the same values, so V-cycles and solves agree bit for bit; the cases cover
a tail below tiled levels, 8x8 blocks, and a hierarchy that lies entirely in
the tail (its first level is the finest, read from the caller's residual)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from tpagmg import BlockTreeMesh, EllipticSolver, MultigridOptions, PoissonOperator, solve  # noqa: E402
from tpagmg import workloads as W  # noqa: E402
import reference_cases as RC  # noqa: E402

CASES = {
    "droplet_l2": (W.droplet_spec(levels=2), 64, True),
    "droplet_l4": (W.droplet_spec(levels=4), 64, True),
    "techref_amr32_b8": (RC.techref_amr(32), 64, False),
    "two_level_b4_all_tail": (RC.two_level_spec(4), 8, False),
}


def build(name):
    spec, coarse, droplet = CASES[name]
    m = BlockTreeMesh(**spec)
    kappa = W.droplet_inputs(m)[1] if droplet else np.ones(m.nfaces)
    return m, EllipticSolver(PoissonOperator(m, kappa), multigrid=MultigridOptions(coarse_size=coarse))


@pytest.mark.parametrize("name", list(CASES))
def test_staged_tail_equals_global_tail(name, monkeypatch):
    m, s = build(name)
    rng = np.random.default_rng(12)
    vol = m.cell_volumes()
    r = rng.standard_normal(m.ncells) * vol
    r -= vol * np.sum(r) / np.sum(vol)
    rhs = W.gaussian_rhs(m, 3)
    out = {}
    for staged in (True, False):
        if staged:
            monkeypatch.setenv("TPAGMG_TAIL_SMEM", "1")
        else:
            monkeypatch.delenv("TPAGMG_TAIL_SMEM", raising=False)
        s.set_tuning()  # rebuild the views under the environment
        zs = [s.vcycle(r, precision=p) for p in ("fp64", "mixed", "fp64")]
        x = np.zeros(m.ncells)
        st = solve(x, s, rhs, rtol=1e-10, precision="mixed")
        out[staged] = (zs, x, st.cycles)
    monkeypatch.delenv("TPAGMG_TAIL_SMEM", raising=False)
    s.set_tuning()
    for a, b in zip(out[True][0], out[False][0]):
        assert np.array_equal(a, b)
    assert np.array_equal(out[True][0][0], out[True][0][2])  # repeatable
    assert out[True][2] == out[False][2] and np.array_equal(out[True][1], out[False][1])
