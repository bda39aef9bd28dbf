"""Oracle (test infrastructure only): CPU restatement of the inverse face
metric K (the face Riesz map) of TwoPhaseAMR.jl's pressure gradient.

Reference (ronaldremmerswaal/TwoPhaseAMR.jl):
  src/operators/gradient.jl:97-158   `_tangential_centre_offset`, `_face_displacement`
  src/operators/gradient.jl:160-171  `_vertex_key`
  src/operators/gradient.jl:194-232  `_local_inverse_metric` (vertex-patch dense metric)
  src/operators/gradient.jl:234-267  `_cached_local_inverse_metric!` (descriptor cache)
  src/operators/gradient.jl:269-292  `_physical_vertex`, `_append_boundary_patch_metric!`
  src/operators/gradient.jl:294-367  `_assemble_inverse_metric` (patch order, COO sum)
  src/operators/gradient.jl:369-393  `_is_diagonal`, `_metric_storage`

Vertex keys are taken on the lattice of the finest active level; the reference
takes them on the refinement-ceiling lattice and shifts them down to the same
lattice (gradient.jl:311-330), so the patch order is the same.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def face_displacements(mesh):
    """`_face_displacement` (gradient.jl:150-158): normal = mean cell width,
    tangential = integer lattice centre offset times half the finest spacing."""
    lattice = mesh.lattice_size()
    mlx, mly, msx, msy = mesh.cell_lattice_bounds(mesh.face_minus, lattice)
    plx, ply, psx, psy = mesh.cell_lattice_bounds(mesh.face_plus, lattice)
    ax = mesh.face_axis
    bm = mesh.face_minus // (mesh.block_size[0] * mesh.block_size[1])
    bp = mesh.face_plus // (mesh.block_size[0] * mesh.block_size[1])
    a0 = ax - 1
    normal = (mesh.spacing[bm, a0] + mesh.spacing[bp, a0]) / 2
    t = 2 - ax  # tangential axis, 0-based
    plow = np.where(t == 0, plx, ply); pscale = np.where(t == 0, psx, psy)
    mlow = np.where(t == 0, mlx, mly); mscale = np.where(t == 0, msx, msy)
    offset = 2 * plow + pscale - 2 * mlow - mscale
    lat_t = np.where(t == 0, lattice[0], lattice[1])
    per_t = np.where(t == 0, mesh.periodic[0], mesh.periodic[1])
    period = 2 * lat_t
    offset = np.where(per_t & (offset > lat_t), offset - period, offset)
    offset = np.where(per_t & (offset < -lat_t), offset + period, offset)
    finest = np.where(t == 0, mesh.extent[0] / lattice[0], mesh.extent[1] / lattice[1])
    tangential = offset * (finest / 2)
    dx = np.where(ax == 1, normal, tangential)
    dy = np.where(ax == 1, tangential, normal)
    return dx, dy


def local_inverse_metric(axes, areas, dx, dy):
    """`_local_inverse_metric` (gradient.jl:194-232) for one vertex patch."""
    n = len(axes)
    if n <= 2:
        raise ValueError("a periodic vertex patch must contain at least three faces")
    moments = np.zeros((n, 2))
    normals = np.zeros((n, 2))
    for r in range(n):
        moments[r, 0] = areas[r] * dx[r]
        moments[r, 1] = areas[r] * dy[r]
        normals[r, axes[r] - 1] = 0.5
    mn = moments.T @ normals
    mn = (mn + mn.T) / 2
    if not (mn[0, 0] > 0 and np.linalg.det(mn) > 0):
        raise ValueError("degenerate vertex patch in gradient construction")
    consistent = normals @ np.linalg.solve(mn, normals.T)
    gram = moments.T @ moments
    projector = np.eye(n) - moments @ np.linalg.solve(gram, moments.T)
    stabilization = np.trace(consistent) / (n - 2)
    local = consistent + stabilization * projector
    return (local + local.T) / 2


def assemble_inverse_metric(mesh):
    """`_assemble_inverse_metric` (gradient.jl:294-367).  Returns the CSC matrix K
    (explicit zeros dropped) and whether it is diagonal (`_metric_storage`)."""
    nf = mesh.nfaces
    lattice = mesh.lattice_size()
    normal, lo, hi = mesh.face_lattice_geometry(lattice)
    dx, dy = face_displacements(mesh)
    areas = mesh.face_area
    axes = mesh.face_axis
    # endpoint keys in face order (endpoint 1 = lo, endpoint 2 = hi)
    kx = np.empty(2 * nf, dtype=np.int64); ky = np.empty(2 * nf, dtype=np.int64)
    for e, tang in ((0, lo), (1, hi)):
        vi = np.where(axes == 1, normal, tang)
        vj = np.where(axes == 1, tang, normal)
        if mesh.periodic[0]:
            vi = vi % lattice[0]
        if mesh.periodic[1]:
            vj = vj % lattice[1]
        kx[e::2] = vi; ky[e::2] = vj
    # two stable counting sorts: by second key, then by first key
    order = np.lexsort((np.arange(2 * nf), ky, kx))
    rows, cols, vals = [], [], []
    cache = {}
    pos = 0
    total = 2 * nf
    okx = kx[order]; oky = ky[order]
    while pos < total:
        stop = pos + 1
        while stop < total and okx[stop] == okx[pos] and oky[stop] == oky[pos]:
            stop += 1
        faces = [int(order[k]) >> 1 for k in range(pos, stop)]
        vx, vy = int(okx[pos]), int(oky[pos])
        pos = stop
        physical = ((not mesh.periodic[0] and (vx == 0 or vx == lattice[0])) or
                    (not mesh.periodic[1] and (vy == 0 or vy == lattice[1])))
        if physical or len(faces) <= 2:
            for f in faces:
                nd = abs(dx[f] if axes[f] == 1 else dy[f])
                if not nd > 0:
                    raise ValueError("degenerate face beside a physical boundary")
                rows.append(f); cols.append(f); vals.append(1.0 / (2.0 * areas[f] * nd))
            continue
        scale = max(max(areas[f], abs(dx[f]), abs(dy[f])) for f in faces)
        desc = lambda f: (int(axes[f]), areas[f] / scale, dx[f] / scale, dy[f] / scale)
        faces.sort(key=desc)
        key = tuple(desc(f) for f in faces)
        normalized = cache.get(key)
        if normalized is None:
            normalized = local_inverse_metric([int(axes[f]) for f in faces], [areas[f] for f in faces],
                                              [dx[f] for f in faces], [dy[f] for f in faces]) * (scale * scale)
            cache[key] = normalized
        local = normalized / (scale * scale)
        for c, cf in enumerate(faces):
            for r, rf in enumerate(faces):
                rows.append(rf); cols.append(cf); vals.append(local[r, c])
    acc = {}
    for r, c, v in zip(rows, cols, vals):
        k = (r, c)
        acc[k] = acc[k] + v if k in acc else v
    items = [(r, c, v) for (r, c), v in acc.items() if v != 0.0]
    r = np.array([t[0] for t in items], dtype=np.int64)
    c = np.array([t[1] for t in items], dtype=np.int64)
    v = np.array([t[2] for t in items], dtype=np.float64)
    K = sp.csc_matrix((v, (r, c)), shape=(nf, nf))
    K.sort_indices()
    diagonal = bool(np.all(r == c))
    if diagonal:
        d = K.diagonal()
        if not np.all(d > 0):
            raise ValueError("gradient Riesz map has a non-positive diagonal")
    return K, diagonal, len(cache)
