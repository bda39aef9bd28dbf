"""CPU checks of the library's host-side set-up against the oracle (bit-exact
integer maps), and of the C-ABI surface.  No device computation runs here."""
import pathlib
import re

import numpy as np
import pytest

from oracle.mesh import block_tree_mesh
from oracle.operator import PoissonOperator as OOp
from oracle.multigrid import MultigridOptions as OMG, TreeGeometricMultigrid

from tpagmg import BlockTreeMesh, EllipticSolver, LinearSolverOptions, MultigridOptions, PoissonOperator
from tpagmg import _lib
from tpagmg import workloads as W

ROOT = pathlib.Path(__file__).resolve().parents[1]


def test_library_exports_every_declared_symbol():
    header = (ROOT / "include" / "tpagmg.h").read_text()
    declared = set(re.findall(r"\b(tpa_[a-z_]+)\s*\(", header))
    assert len(declared) >= 20
    lib = _lib.lib()
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(_lib.SIGNATURES)


def two_level(bs):
    return dict(block_size=(bs, bs), max_level=2,
                refine=lambda k, o, e: k[0] == 0 or (k[0] == 1 and k[1] == 0 and k[2] == 0))


SPECS = {
    "two_level_b4": (two_level(4), 8, None),
    "two_level_b8": (two_level(8), 8, None),
    "pruned_varcoef": (dict(block_size=(8, 8), max_level=3,
                            refine=lambda k, o, e: k[0] == 0 or (k[0] < 3 and o[0] < 0.5 and o[1] < 0.5)),
                       64, lambda m: np.exp(0.4 * np.sin(np.arange(m.nfaces) + 1.0))),
    "droplet_l2": (W.droplet_spec(levels=2), 64, None),
    **{f"walls_{p[0]}_{p[1]}": (dict(base_mesh=(16, 16), block_size=(4, 4), origin=(-1.0, 0.25), extent=(2.0, 1.5),
                                     periodic=p), 16, None)
       for p in ((True, True), (True, False), (False, True), (False, False))},
    "unbalanced_leaves": (dict(base_mesh=(32, 32), block_size=(4, 4), max_level=3,
                               refine=lambda k, o, e: k == (0, 3, 3) or k == (1, 7, 7) or k == (2, 14, 15)), 16, None),
}


@pytest.mark.parametrize("name", list(SPECS))
def test_host_setup_bit_exact(name):
    spec, coarse, coef = SPECS[name]
    m = BlockTreeMesh(**spec)
    o = block_tree_mesh(**spec)
    assert np.array_equal(m.keys, np.array(o.keys))
    for a, b in ((m.face_minus, o.face_minus), (m.face_plus, o.face_plus), (m.face_axis, o.face_axis),
                 (m.bface_cell, o.bface_cell), (m.bface_axis, o.bface_axis), (m.bface_side, o.bface_side)):
        assert np.array_equal(a, b)
    assert np.array_equal(m.face_area, o.face_area)
    assert np.array_equal(m.bface_area, o.bface_area)
    assert np.array_equal(m.volume, o.volume) and np.array_equal(m.spacing, o.spacing)
    kappa = np.ones(m.nfaces) if coef is None else coef(m)
    s = EllipticSolver(PoissonOperator(m, kappa), multigrid=MultigridOptions(coarse_size=coarse))
    oo = OOp(o, kappa)
    mg = TreeGeometricMultigrid(oo, OMG(coarse_size=coarse))
    assert s.level_sizes() == mg.level_sizes
    for lev in range(len(mg.levels) - 1):
        assert np.array_equal(s.level_owners(lev), mg.owners[lev])
        sw, tw, nc = s.level_info(lev)
        assert sw == pytest.approx(mg.levels[lev].weight, rel=1e-14)
        assert tw == pytest.approx(mg.transfer_weights[lev], rel=1e-13)
        assert nc == len(mg.levels[lev].component_volumes)
    for lev, op in enumerate(mg.operators):
        assert np.allclose(s.level_face_coefficients(lev, op.mesh.nfaces), op.face_coefficient, rtol=1e-15, atol=0)


def test_options_mirror_reference_validation():
    with pytest.raises(TypeError):
        MultigridOptions(coarse_size=1.5)
    with pytest.raises(ValueError):
        MultigridOptions(coarse_size=0)
    with pytest.raises(ValueError):
        MultigridOptions(pre_sweeps=-1)
    with pytest.raises(ValueError):
        LinearSolverOptions(preconditioner="bogus")
    with pytest.raises(ValueError):
        LinearSolverOptions(krylov="cg")
    m = BlockTreeMesh(**two_level(4))
    with pytest.raises(ValueError):
        EllipticSolver(PoissonOperator(m), multigrid=MultigridOptions(pre_sweeps=1, post_sweeps=3))
    with pytest.raises(ValueError):
        PoissonOperator(m, -np.ones(m.nfaces))
    with pytest.raises(ValueError):
        PoissonOperator(m, np.ones(m.nfaces + 1))


def test_device_entry_points_fail_loudly_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    m = BlockTreeMesh(**two_level(4))
    s = EllipticSolver(PoissonOperator(m))
    with pytest.raises(_lib.TpaError) as e:
        s.apply(np.zeros(m.ncells))
    assert e.value.code == _lib.TPA_ERR_CUDA


def test_invalid_mesh_arguments():
    with pytest.raises(ValueError):
        BlockTreeMesh(block_size=(3, 3))
    with pytest.raises(_lib.TpaError):
        BlockTreeMesh(base_mesh=(32, 32), block_size=(16, 16), leaves=[(0, 0, 0)])


def test_noalloc_norms_reject_sizes_before_any_cuda_call():
    """tpa_residual_norms_noalloc checks its size (1 <= n <= 2^31 - 1, the
    library's 32-bit cell indices) and its pointers before touching the
    device, so the rejection holds on a host without a GPU.  The pointers
    passed here are never dereferenced."""
    import ctypes as C
    lib = _lib.lib()
    ctx = _lib.Context(0)  # no CUDA call until the first device operation
    out = np.zeros(2)
    fake = C.c_void_p(256)
    for n in (2 ** 31, 2 ** 40, 0, -5):
        st = lib.tpa_residual_norms_noalloc(ctx.handle, fake, fake, n, out.ctypes.data_as(C.POINTER(C.c_double)))
        assert st == _lib.TPA_ERR_INVALID_ARG
        assert b"[1, 2147483647]" in lib.tpa_last_error(ctx.handle)
    st = lib.tpa_residual_norms_noalloc(ctx.handle, None, fake, 10, out.ctypes.data_as(C.POINTER(C.c_double)))
    assert st == _lib.TPA_ERR_INVALID_ARG
    # without a context the status alone reports the rejection
    assert lib.tpa_residual_norms_noalloc(None, fake, fake, 2 ** 31, out.ctypes.data_as(C.POINTER(C.c_double))) \
        == _lib.TPA_ERR_INVALID_ARG
