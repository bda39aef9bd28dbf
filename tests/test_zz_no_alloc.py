"""The allocation-free residual norms.

`tpa_residual_norms_noalloc` serves callers that cannot call cudaMalloc
(device memory owned by a pool or arena that must not be bypassed, hosts that
forbid runtime allocation): its scratch is a static device array.  It must give
the same norms as the context entry point `tpa_residual_norms`, call after
call, and the oracle's `_integrated_residual_norms` on the inputs the context
entry point cannot take (zero volumes, a single cell, a NaN).  This file is
collected last so that a run stopping at its first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from tpagmg import BlockTreeMesh, EllipticSolver, PoissonOperator, _lib  # noqa: E402
from tpagmg import workloads as W  # noqa: E402
from oracle.krylov import integrated_norms  # noqa: E402


def _call(lib, handle, r, vol, n):
    out = np.full(2, -1.0)
    status = lib.tpa_residual_norms_noalloc(handle, C.c_void_p(r.data_ptr()), C.c_void_p(vol.data_ptr()), n,
                                            out.ctypes.data_as(C.POINTER(C.c_double)))
    assert status == _lib.TPA_OK, lib.tpa_last_error(handle)
    return out


def test_noalloc_norms_match_context_entry_point_twice():
    import torch
    mesh = BlockTreeMesh(**W.droplet_spec(levels=2))
    _, kappa, _ = W.droplet_inputs(mesh)
    solver = EllipticSolver(PoissonOperator(mesh, kappa))
    vol = torch.from_numpy(mesh.cell_volumes()).cuda()
    lib = _lib.lib()
    for seed in (1, 2):  # two calls in a row share (and reuse) the static scratch
        r = np.random.default_rng(seed).standard_normal(mesh.ncells) * mesh.cell_volumes()
        rd = torch.from_numpy(r).cuda()
        ref = solver.residual_norms_device(rd.data_ptr())
        out = _call(lib, solver.ctx.handle, rd, vol, mesh.ncells)
        # the same tolerance as the device-versus-oracle norm test
        assert out[0] == pytest.approx(ref[0], rel=1e-12)
        assert out[1] == pytest.approx(ref[1], rel=1e-15)
    # a NaN residual: both entry points report NaN norms (the reference's
    # canonical NaN maximum, cycles.jl:230-260)
    r[7] = np.nan
    rd = torch.from_numpy(r).cuda()
    ref = solver.residual_norms_device(rd.data_ptr())
    out = _call(lib, solver.ctx.handle, rd, vol, mesh.ncells)
    assert np.isnan(ref[1]) and np.isnan(out[1]) and np.isnan(out[0])


def test_noalloc_norms_zero_volumes_and_small_sizes():
    """Cells of zero volume are skipped, and sizes far below the fixed grid
    (most of its blocks fold zero partials) agree with the oracle."""
    import torch
    lib = _lib.lib()
    rng = np.random.default_rng(3)
    for n in (1, 5, 1000, 300_001):
        vol = rng.uniform(0.5, 2.0, n)
        vol[rng.random(n) < 0.2] = 0.0
        vol[0] = 1.0
        r = rng.standard_normal(n)
        out = _call(lib, None, torch.from_numpy(r).cuda(), torch.from_numpy(vol).cuda(), n)
        l2, mx = integrated_norms(r, vol)
        assert out[0] == pytest.approx(l2, rel=1e-12)
        assert out[1] == mx


def test_noalloc_norms_make_no_device_allocation():
    import torch
    lib = _lib.lib()
    n = 1 << 20
    r = torch.randn(n, dtype=torch.float64, device="cuda")
    vol = torch.ones(n, dtype=torch.float64, device="cuda")
    first = _call(lib, None, r, vol, n)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(20):
        out = _call(lib, None, r, vol, n)
        assert np.array_equal(out, first)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before


def test_noalloc_rejects_sizes_beyond_the_maximum():
    import torch
    mesh = BlockTreeMesh(**W.droplet_spec(levels=1))
    solver = EllipticSolver(PoissonOperator(mesh))
    v = torch.ones(4, dtype=torch.float64, device="cuda")
    out = np.zeros(2)
    lib = _lib.lib()
    for n in (2 ** 31, 0):
        status = lib.tpa_residual_norms_noalloc(solver.ctx.handle, C.c_void_p(v.data_ptr()), C.c_void_p(v.data_ptr()),
                                                n, out.ctypes.data_as(C.POINTER(C.c_double)))
        assert status == _lib.TPA_ERR_INVALID_ARG
        assert b"2147483647" in lib.tpa_last_error(solver.ctx.handle)
