"""Seeded synthetic pressure-solve workloads (no dataset is involved).

Each workload is a mesh specification, face coefficients and a strong-form
right-hand side, generated once on the host with numpy's counter-based Philox
bit generator and shared by every solver that is compared on it.

  taylor_green_128   128x128 periodic cells on [0, 2pi]^2 (8x8 blocks of 16x16),
                     kappa = 1, RHS = discrete divergence of
                     u = (sin x cos y, -cos x sin y) + N(0, 1e-3) noise, zero mean
  droplet_amr        unit square, free-slip walls, 4x4 blocks of 16x16 refined 4
                     levels (finest h = 1/1024) in a band of 8 finest cells around
                     the circle |x - (0.5, 0.6)| = 0.15; density 1000 inside and 1
                     outside (kappa = 1/rho_f), CGFM surface-tension RHS
                     L psi / V, psi = sigma * curvature * [c > 1/2] with sigma =
                     0.072 and curvature 1/0.15, plus N(0, 1) noise, zero mean
  uniform_2048       2048x2048 periodic cells on the unit square (128x128 blocks),
                     kappa = 1, RHS N(0, 1), zero mean
"""
from __future__ import annotations

import math

import numpy as np

SEEDS = {"taylor_green_128": 101, "droplet_amr": 202, "uniform_2048": 303, "batch": 404, "adjoint": 505}


def rng(seed):
    return np.random.Generator(np.random.Philox(seed))


def zero_mean(values, volumes):
    return values - np.sum(values * volumes) / np.sum(volumes)


# ---- mesh specifications ------------------------------------------------------

def taylor_green_spec(n=128, block=16):
    return dict(base_mesh=(n, n), block_size=(block, block), extent=(2 * math.pi, 2 * math.pi),
                periodic=(True, True))


def uniform_spec(n=2048, block=16):
    return dict(base_mesh=(n, n), block_size=(block, block), extent=(1.0, 1.0), periodic=(True, True))


def circle_band_refine(center=(0.5, 0.6), radius=0.15, band=8 / 1024):
    """Refine every block whose box lies within `band` of the circle (box-to-curve
    distance: zero when the circle crosses the box)."""
    cx, cy = center

    def refine(key, origin, extent):
        x0, y0 = origin
        x1, y1 = origin[0] + extent[0], origin[1] + extent[1]
        dmin = math.hypot(max(x0 - cx, 0.0, cx - x1), max(y0 - cy, 0.0, cy - y1))
        dmax = max(math.hypot(x - cx, y - cy) for x in (x0, x1) for y in (y0, y1))
        if dmin <= radius <= dmax:
            return True
        d = dmin - radius if radius < dmin else radius - dmax
        return d <= band
    return refine


def droplet_spec(levels=4, base=64, block=16, radius=0.15, center=(0.5, 0.6)):
    finest = 1.0 / (base << levels)
    return dict(base_mesh=(base, base), block_size=(block, block), extent=(1.0, 1.0), periodic=(False, False),
                max_level=levels, refine=circle_band_refine(center, radius, 8 * finest))


# ---- circle fractions (exact disk / rectangle intersection areas) --------------

def _chord_integral(x0, x1, cx, cy, r, y0, y1):
    """Exact area of the disk (cx, cy, r) inside [x0, x1] x [y0, y1]."""
    a, b = max(x0, cx - r), min(x1, cx + r)
    if a >= b:
        return 0.0
    s = lambda x: math.sqrt(max(r * r - (x - cx) ** 2, 0.0))
    F = lambda x: 0.5 * ((x - cx) * s(x) + r * r * math.asin(max(-1.0, min(1.0, (x - cx) / r))))
    cuts = {a, b}
    for yy in (y0, y1):
        d = abs(yy - cy)
        if d < r:
            w = math.sqrt(r * r - d * d)
            for xx in (cx - w, cx + w):
                if a < xx < b:
                    cuts.add(xx)
    pts = sorted(cuts)
    area = 0.0
    for lo, hi in zip(pts[:-1], pts[1:]):
        m = 0.5 * (lo + hi)
        top_s = cy + s(m) < y1
        bot_s = cy - s(m) > y0
        top_full = cy + s(m) >= y1
        bot_full = cy - s(m) <= y0
        if cy + s(m) <= y0 or cy - s(m) >= y1:
            continue
        # integral of min(y1, cy + s) - max(y0, cy - s)
        if top_full and bot_full:
            area += (y1 - y0) * (hi - lo)
        elif top_s and bot_s:
            area += 2 * (F(hi) - F(lo))
        elif top_s and bot_full:
            area += (cy - y0) * (hi - lo) + (F(hi) - F(lo))
        else:  # top_full and bot_s
            area += (y1 - cy) * (hi - lo) + (F(hi) - F(lo))
    return area


def circle_fractions(mesh, center=(0.5, 0.6), radius=0.15):
    """Liquid (inside) area fraction of every cell."""
    x, y = mesh.cell_centers()
    nx, ny = mesh.block_size
    hx = np.repeat(mesh.spacing[:, 0], nx * ny)
    hy = np.repeat(mesh.spacing[:, 1], nx * ny)
    cx, cy = center
    dnear = np.hypot(np.maximum(np.abs(x - cx) - hx / 2, 0), np.maximum(np.abs(y - cy) - hy / 2, 0))
    dfar = np.hypot(np.abs(x - cx) + hx / 2, np.abs(y - cy) + hy / 2)
    frac = np.where(dfar <= radius, 1.0, 0.0)
    cut = np.nonzero((dnear < radius) & (dfar > radius))[0]
    for c in cut:
        x0, x1 = x[c] - hx[c] / 2, x[c] + hx[c] / 2
        y0, y1 = y[c] - hy[c] / 2, y[c] + hy[c] / 2
        frac[c] = min(1.0, max(0.0, _chord_integral(x0, x1, cx, cy, radius, y0, y1) / (hx[c] * hy[c])))
    return frac


# ---- right-hand sides ------------------------------------------------------------

def taylor_green_rhs(mesh, seed=SEEDS["taylor_green_128"], noise=1e-3):
    """Discrete divergence (cell_advection.jl:205-220) of the face-sampled
    Taylor-Green field plus N(0, noise) per cell, volume mean removed."""
    cx, cy = mesh.face_centers()
    u = np.where(mesh.face_axis == 1, np.sin(cx) * np.cos(cy), -np.cos(cx) * np.sin(cy))
    flux = u * mesh.face_area
    vol = mesh.cell_volumes()
    div = np.zeros(mesh.ncells)
    np.add.at(div, mesh.face_minus, flux / vol[mesh.face_minus])
    np.add.at(div, mesh.face_plus, -flux / vol[mesh.face_plus])
    div += noise * rng(seed).standard_normal(mesh.ncells)
    return zero_mean(div, vol)


def gaussian_rhs(mesh, seed):
    vol = mesh.cell_volumes()
    return zero_mean(rng(seed).standard_normal(mesh.ncells), vol)


def droplet_inputs(mesh, density=(1000.0, 1.0), sigma=0.072, radius=0.15, center=(0.5, 0.6)):
    """Cell fractions, face coefficients kappa = 1/rho_f and the potential psi of
    the CGFM surface-tension jump (psi_p - psi_m = jump / |f|)."""
    from .operator import mixture_density
    frac = circle_fractions(mesh, center, radius)
    kappa = 1.0 / mixture_density(mesh, frac, density)
    psi = sigma * (1.0 / radius) * (frac > 0.5).astype(np.float64)
    return frac, kappa, psi


def droplet_rhs(mesh, L_psi, seed=SEEDS["droplet_amr"], noise=1.0):
    """Strong RHS (L psi)/V + N(0, noise), volume mean removed; `L_psi` is the
    integrated operator applied to psi."""
    vol = mesh.cell_volumes()
    b = L_psi / vol
    if noise:
        b = b + noise * rng(seed).standard_normal(mesh.ncells)
    return zero_mean(b, vol)


# ---- batched uneven solves ------------------------------------------------------

def batch_problems(count=256, seed=SEEDS["batch"]):
    """Parameters of `count` independent two-phase problems on the unit square
    with free-slip walls and base 2x2 blocks of 16x16 cells: tree depth
    U{2..6}, circle radius U[0.05, 0.3], centre U[0.3, 0.7]^2, density ratio
    from {10, 100, 1000} (heavy phase inside), RHS seed 404000 + k."""
    g = rng(seed)
    out = []
    for k in range(count):
        depth = int(g.integers(2, 7))
        radius = float(g.uniform(0.05, 0.3))
        center = (float(g.uniform(0.3, 0.7)), float(g.uniform(0.3, 0.7)))
        ratio = float(g.choice([10.0, 100.0, 1000.0]))
        out.append(dict(index=k, depth=depth, radius=radius, center=center, ratio=ratio, rhs_seed=seed * 1000 + k))
    return out


def batch_spec(problem, base=32, block=16):
    """Mesh of one batched problem: refined to its depth in a band of 8 finest
    cells around its circle."""
    finest = 1.0 / (base << problem["depth"])
    return dict(base_mesh=(base, base), block_size=(block, block), extent=(1.0, 1.0), periodic=(False, False),
                max_level=problem["depth"],
                refine=circle_band_refine(problem["center"], problem["radius"], 8 * finest))


def batch_inputs(mesh, problem):
    """Face coefficients kappa = 1/rho_f (rho = ratio inside, 1 outside) and the
    zero-mean N(0, 1) strong right-hand side of one batched problem."""
    from .operator import mixture_density
    frac = circle_fractions(mesh, problem["center"], problem["radius"])
    kappa = 1.0 / mixture_density(mesh, frac, (problem["ratio"], 1.0))
    return kappa, gaussian_rhs(mesh, problem["rhs_seed"])
