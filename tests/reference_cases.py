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


# Chapter 11 fixtures of the technical reference (docs/techref/figures/solvers.jl
# of the reference): walls, 8x8 blocks, a drop circle and a deterministic noise RHS.
TECHREF_CENTRE = (0.513, 0.468)   # SOLV_DROP, solvers.jl:19
TECHREF_RADIUS = 0.2371
TECHREF_BAND = 0.02
TECHREF_DENSITY = (1000.0, 1.0)   # SOLV_DENSITY, solvers.jl:16


def techref_noise(n):
    """`solv_noise(index)` (solvers.jl:24) for the 1-based cell indices 1..n."""
    idx = np.arange(1, n + 1, dtype=np.float64)
    v = np.sin(12.9898 * idx) * 43758.5453
    return v - np.floor(v) - 0.5


def techref_uniform(n):
    """`solv_uniform(n)` (solvers.jl:26-28)."""
    return dict(base_mesh=(n, n), block_size=(8, 8), periodic=(False, False))


def _techref_near_circle(origin, extent):
    """`solv_near_circle` (solvers.jl:31-38): the block box comes within the band of the circle."""
    xs = (origin[0], origin[0] + extent[0])
    ys = (origin[1], origin[1] + extent[1])
    cx, cy = TECHREF_CENTRE
    nearest = np.hypot(min(max(cx, xs[0]), xs[1]) - cx, min(max(cy, ys[0]), ys[1]) - cy)
    farthest = max(np.hypot(x - cx, y - cy) for x in xs for y in ys)
    return nearest - TECHREF_BAND <= TECHREF_RADIUS <= farthest + TECHREF_BAND


def techref_amr(n, levels=2):
    """`solv_amr(n)` (solvers.jl:40-45)."""
    return dict(base_mesh=(n, n), block_size=(8, 8), periodic=(False, False), max_level=levels,
                refine=lambda k, o, e: _techref_near_circle(o, e))


TECHREF_CASES = {
    "uniform64": (techref_uniform, 64, False), "uniform128": (techref_uniform, 128, False),
    "uniform256": (techref_uniform, 256, False), "amr32": (techref_amr, 32, False),
    "amr64": (techref_amr, 64, False), "drop128": (techref_uniform, 128, True),
    "dropamr": (techref_amr, 64, True),
}
TECHREF_VCYCLE_CASES = {
    "uniform16": (techref_uniform, 16, False), "uniform32": (techref_uniform, 32, False),
    "amr16": (techref_amr, 16, False), "drop32": (techref_uniform, 32, True),
}
