"""The allocation-free residual norms.

`tpa_residual_norms_noalloc` serves callers that cannot call cudaMalloc (code
under CUDA graph capture, pool- or arena-owned device memory, hosts that forbid
runtime allocation): its scratch is a static device array.  It must give the
same norms as the context entry point `tpa_residual_norms`, call after call.
This file is collected last so that a run stopping at its first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from tpagmg import BlockTreeMesh, EllipticSolver, PoissonOperator, _lib  # noqa: E402
from tpagmg import workloads as W  # noqa: E402


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
        out = np.zeros(2)
        status = lib.tpa_residual_norms_noalloc(solver.ctx.handle, C.c_void_p(rd.data_ptr()),
                                                C.c_void_p(vol.data_ptr()), mesh.ncells,
                                                out.ctypes.data_as(C.POINTER(C.c_double)))
        assert status == _lib.TPA_OK, lib.tpa_last_error(solver.ctx.handle)
        # the same tolerance as the device-versus-oracle norm test
        assert out[0] == pytest.approx(ref[0], rel=1e-12)
        assert out[1] == pytest.approx(ref[1], rel=1e-15)


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
