"""Inputs of reference testsets restated by the oracle and GPU tests
(test/operators/poisson.jl of ronaldremmerswaal/TwoPhaseAMR.jl).  Test
infrastructure: mesh specs and fields only, no solver."""
import numpy as np


def chain_spec():
    """:672-681: an 8x8-cell base of 4x4 blocks refined along the diagonal to level 3."""
    return dict(base_mesh=(8, 8), block_size=(4, 4), max_level=3,
                refine=lambda k, o, e: (k[0] == 0 and k[1] == 0 and k[2] == 0) or
                (k[0] == 1 and k[1] == 1 and k[2] == 1) or (k[0] == 2 and k[1] == 2 and k[2] == 2))


def chain_exact(x, y):
    """:699-702."""
    return np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) + 0.2 * np.cos(np.pi * (4 * x - 2 * y)) \
        + 0.1 * np.sin(4 * np.pi * y)


def two_level_spec(block):
    return dict(block_size=(block, block), max_level=2,
                refine=lambda k, o, e: k[0] == 0 or (k[0] == 1 and k[1] == 0 and k[2] == 0))


def deep_spec():
    """:834-839: 8x8 blocks refined to level 4 in the lower-left quarter."""
    return dict(block_size=(8, 8), max_level=4,
                refine=lambda k, o, e: k[0] == 0 or (k[0] < 4 and o[0] < 0.5 and o[1] < 0.5))


def deep_rhs(x, y):
    """:840-845."""
    return 8 * np.pi ** 2 * np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y) + 2 * np.pi ** 2 * np.sin(2 * np.pi * (x + y))


def harmonic_face_coefficients(mesh, cell_value):
    """`harmonic_face_coefficients` (src/operators/elliptic.jl:9-23): the
    distance-weighted harmonic mean of the two cell values."""
    nx, ny = mesh.block_size
    a = mesh.face_axis.astype(np.int64) - 1
    dm = mesh.spacing[mesh.face_minus // (nx * ny), a] / 2
    dp = mesh.spacing[mesh.face_plus // (nx * ny), a] / 2
    cm, cp = cell_value[mesh.face_minus], cell_value[mesh.face_plus]
    return (dm + dp) / (dm / cm + dp / cp)
