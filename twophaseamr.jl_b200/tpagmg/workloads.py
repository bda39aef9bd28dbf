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
  capillary_wave     the mesh of examples/07_capillary_wave (8x24 roots of 8x8 on
                     [0, 1] x [-1.5, 1.5], periodic in x) refined `max_level` levels
                     in a band around y = 0.25 + 0.01 cos(2 pi x), density 1 below
                     and 1e-3 above; with it, a seeded synthetic CMDGFM system of
                     the reference's block structure (`cmdgfm_system`)
"""
from __future__ import annotations

import math

import numpy as np

SEEDS = {"taylor_green_128": 101, "droplet_amr": 202, "uniform_2048": 303, "batch": 404, "adjoint": 505,
         "cmdgfm": 606}


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


# ---- the capillary wave and a CMDGFM system on it ---------------------------------

WAVE_LEVEL, WAVE_AMPLITUDE = 0.25, 0.01


def wave_height(x, amplitude=WAVE_AMPLITUDE):
    return WAVE_LEVEL + amplitude * np.cos(2 * np.pi * x)


def capillary_wave_spec(max_level=4, amplitude=WAVE_AMPLITUDE, band_cells=4):
    """examples/07_capillary_wave/capillary_wave.jl:40-44: 8 x 24 roots of 8 x 8
    cells on [0, 1] x [-1.5, 1.5], periodic in x; every block within
    `band_cells` finest cells of the interface band is refined, to
    `max_level` (the example refines to the interface indicator's level)."""
    band = band_cells / (64 << max_level)

    def refine(key, origin, extent):
        y0, y1 = origin[1], origin[1] + extent[1]
        return y0 - band <= WAVE_LEVEL + amplitude and y1 + band >= WAVE_LEVEL - amplitude
    return dict(base_mesh=(8, 24), block_size=(8, 8), origin=(0.0, -1.5), extent=(1.0, 3.0),
                periodic=(True, False), max_level=max_level, refine=refine)


def wave_fractions(mesh, amplitude=WAVE_AMPLITUDE, samples=16):
    """Liquid (below the interface) area fraction of every cell: the height
    function averaged over `samples` abscissae of the cell."""
    x, y = mesh.cell_centers()
    nx, ny = mesh.block_size
    hx = np.repeat(mesh.spacing[:, 0], nx * ny)
    hy = np.repeat(mesh.spacing[:, 1], nx * ny)
    off = (np.arange(samples) + 0.5) / samples - 0.5
    xs = x[:, None] + off[None, :] * hx[:, None]
    eta = wave_height(xs, amplitude)
    frac = np.clip((eta - (y - hy / 2)[:, None]) / hy[:, None], 0.0, 1.0)
    return frac.mean(axis=1)


def cmdgfm_system(mesh, matrix, kappa, fractions, *, density=(1.0, 1e-3), dt=1e-3, seed=SEEDS["cmdgfm"],
                  theta=0.5, transverse=(0.25, 0.15)):
    """A seeded synthetic CMDGFM system with the block structure that
    `_assemble_cmdgfm_system!` (cmdgfm_projection.jl:1484-1592) produces, and
    its exact solution: returns (CMDGFMSystem, exact).

    * Gauge (common.jl:89-112): one component, anchored at cell 0; the other
      cells are the pressure unknowns, in order.
    * Mixed faces: faces whose two cells lie on different sides of c = 1/2, in
      face order; one jump unknown each.
    * A: the pressure operator's assembled matrix (`matrix`, integrated form)
      without the anchor's row and column.  B: the coupling kappa_f |f| of a
      jump into its two cells' rows, -1 on the minus cell and +1 on the plus
      cell (`_cmdgfm_anchor_residual_defect`, :1866-1877).
    * J: unit diagonal (cmdgfm_projection.jl:1345-1347) with transverse
      couplings -transverse[0] to the next and -transverse[1] to the previous
      mixed face along the interface (face centres within 1.5 h).  C: the
      inference gradient rows, +-theta / h on the face's two cells.
    * The exact solution: pressure P (sin(2 pi x) exp(-|y - 0.25|) + 0.01
      N(0, 1)) with P = rho_max / (2 pi dt)^2, jumps (h_ref / dt^2) 0.1 N(0, 1);
      the right-hand side and the anchor row's are its products.
    * Defect weights dt^2 / V and dt^2 / h; the scaling of
      `_cmdgfm_krylov_scaling!` (:215-235) with the domain length h_ref."""
    import scipy.sparse as sp
    from scipy.spatial import cKDTree
    from .cmdgfm import CMDGFMSystem

    row_ptr, col, val = matrix
    ncells = mesh.ncells
    A = sp.csr_matrix((val, col, row_ptr), shape=(ncells, ncells))
    fr = np.asarray(fractions)
    mixed = np.nonzero((fr[mesh.face_minus] > 0.5) != (fr[mesh.face_plus] > 0.5))[0]
    nxj = len(mixed)
    npr = ncells - 1
    cells = np.arange(1, ncells)
    anchor = 0
    # unknown index of a cell (-1: the anchor)
    idx = np.arange(ncells) - 1
    nxb, nyb = mesh.block_size
    spacing = np.minimum(mesh.spacing[:, 0], mesh.spacing[:, 1])
    hm = spacing[mesh.face_minus[mixed] // (nxb * nyb)]
    hp = spacing[mesh.face_plus[mixed] // (nxb * nyb)]
    h = np.minimum(hm, hp)
    w = np.asarray(kappa)[mixed] * mesh.face_area[mixed]
    m_cell, p_cell = mesh.face_minus[mixed], mesh.face_plus[mixed]
    # B and the anchor's entries
    brow = np.concatenate([m_cell, p_cell])
    bcol = np.concatenate([np.arange(nxj), np.arange(nxj)])
    bval = np.concatenate([-w, w])
    B_full = sp.csr_matrix((bval, (brow, bcol)), shape=(ncells, nxj))
    A_red = A[cells][:, cells]
    B_red = B_full[cells]
    # C on the pressure unknowns (anchor columns dropped)
    crow, ccol, cval = [], [], []
    for k in range(nxj):
        for c_, sgn in ((m_cell[k], 1.0), (p_cell[k], -1.0)):
            if idx[c_] >= 0:
                crow.append(k)
                ccol.append(idx[c_])
                cval.append(sgn * theta / h[k])
    Cm = sp.csr_matrix((cval, (crow, ccol)), shape=(nxj, npr))
    # J: transverse neighbours along the interface
    fx, fy = mesh.face_centers()
    pts = np.stack([fx[mixed] % 1.0, fy[mixed] + 2.0], axis=1)
    jrow, jcol, jval = list(range(nxj)), list(range(nxj)), [1.0] * nxj
    if nxj:
        tree = cKDTree(pts, boxsize=[1.0, 1e9])
        for k in range(nxj):
            for kk in tree.query_ball_point(pts[k], 1.5 * h[k]):
                if kk != k:
                    jrow.append(k)
                    jcol.append(kk)
                    jval.append(-(transverse[0] if kk > k else transverse[1]) / 4.0)
    J = sp.csr_matrix((jval, (jrow, jcol)), shape=(nxj, nxj))
    M = sp.bmat([[A_red, B_red], [Cm, J]], format="csr")
    M.sort_indices()
    x, y = mesh.cell_centers()
    g = rng(seed)
    P = max(density) / (2 * np.pi * dt) ** 2
    p_exact = P * (np.sin(2 * np.pi * x) * np.exp(-np.abs(y - WAVE_LEVEL)) + 0.01 * g.standard_normal(ncells))
    p_exact -= p_exact[anchor]
    h_ref = max(3.0, 1.0)
    xi_exact = (h_ref / dt ** 2) * 0.1 * g.standard_normal(nxj)
    exact = np.concatenate([p_exact[cells], xi_exact])
    rhs = M @ exact
    E = sp.hstack([A[[anchor]][:, cells], B_full[[anchor]]], format="csr")
    E.sort_indices()
    vol = mesh.cell_volumes()
    n = npr + nxj
    weight = np.concatenate([dt ** 2 / vol[cells], dt ** 2 / h])
    rows = np.concatenate([np.full(npr, (dt / h_ref) ** 2), np.full(nxj, dt ** 2 / h_ref)])
    cols = np.concatenate([np.full(npr, max(density) * (h_ref / dt) ** 2), np.full(nxj, h_ref / dt ** 2)])
    system = CMDGFMSystem(np_=npr, row_ptr=M.indptr.astype(np.int64), col=M.indices.astype(np.int32),
                          val=M.data.astype(np.float64), rhs=rhs, pressure_cell=cells.astype(np.int32),
                          pressure_anchor=np.full(npr, anchor, dtype=np.int32), defect_weight=weight,
                          extra_row_ptr=E.indptr.astype(np.int64), extra_col=E.indices.astype(np.int32),
                          extra_val=E.data.astype(np.float64), extra_rhs=E @ exact,
                          extra_weight=np.array([dt ** 2 / vol[anchor]]), row_scale=rows, col_scale=cols)
    assert system.n == n
    return system, exact
