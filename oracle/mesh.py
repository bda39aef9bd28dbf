"""Oracle (test infrastructure only): CPU restatement of TwoPhaseAMR.jl's
block quadtree forest, its leaf order and its face schedules.

This module is a checker. Only `tests/`, `__graft_entry__.smoke()` and the CPU
baseline leg of `bench.py` may import it; the shipped solver never does.

Reference (paths inside ronaldremmerswaal/TwoPhaseAMR.jl):
  src/mesh/topology/mesh.jl:1-30      BlockKey, CellRef, `_cell_index`
  src/mesh/topology/mesh.jl:673-714   `_balance!` (2:1 grading, corners and periodic seams)
  src/mesh/topology/mesh.jl:716-757   `_build_tree`, `_build_root_grid`
  src/mesh/topology/mesh.jl:759-773   `_leaf_blocks` (sort by level, j, i)
  src/mesh/topology/mesh.jl:787-937   `_lattice_sides`, `_match_sides!`, `_push_boundary!`
  src/mesh/topology/mesh.jl:450-485   `_cell_lattice_bounds`, `_face_lattice_geometry`
  src/mesh/topology/mesh.jl:1059-1121 `BlockTreeMesh` constructor

Indices are 0-based here (cell index = block * nx * ny + j * nx + i), which is the
reference's 1-based `_cell_index` shifted by one.  The halo schedule
(`_build_halo_schedule`) is not restated: the pressure solve never reads halos.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Tree:
    """Quadtree forest over a `layout` of level-0 roots (mesh.jl:103-110)."""

    layout: tuple
    origin: tuple
    extent: tuple
    root_extent: tuple
    leaves: set = field(default_factory=set)     # {(level, i, j)}
    internal: set = field(default_factory=set)

    def node_box(self, key):
        """Physical (origin, extent) of a node: RegionTrees halves the parent."""
        level, i, j = key
        if level == 0:
            return ((self.origin[0] + i * self.root_extent[0],
                     self.origin[1] + j * self.root_extent[1]), self.root_extent)
        parent = (level - 1, i >> 1, j >> 1)
        (px, py), (wx, wy) = self.node_box(parent)
        hx, hy = wx / 2, wy / 2
        return ((px + (i & 1) * hx, py + (j & 1) * hy), (hx, hy))

    def split(self, key):
        self.leaves.discard(key)
        self.internal.add(key)
        level, i, j = key
        for cj in (0, 1):
            for ci in (0, 1):
                self.leaves.add((level + 1, 2 * i + ci, 2 * j + cj))

    def leaf_at(self, level, i, j):
        """Leaf covering the level-`level` node box (i, j), if that box lies in
        one leaf of level <= `level`; else None (the region is refined)."""
        for lev in range(0, level + 1):
            key = (lev, i >> (level - lev), j >> (level - lev))
            if key in self.leaves:
                return key
            if key not in self.internal:
                return None
        return None


def build_tree(base_mesh, block_size, origin, extent, max_level, refine):
    """`_build_root_grid` (mesh.jl:716-757): recursive `refine` callback per root."""
    layout = (base_mesh[0] // block_size[0], base_mesh[1] // block_size[1])
    root_extent = (extent[0] / layout[0], extent[1] / layout[1])
    tree = Tree(layout, tuple(origin), tuple(extent), root_extent)

    def visit(key):
        if key[0] >= max_level:
            tree.leaves.add(key)
            return
        box_origin, box_extent = tree.node_box(key)
        if refine(key, box_origin, box_extent):
            tree.internal.add(key)
            level, i, j = key
            for cj in (0, 1):
                for ci in (0, 1):
                    visit((level + 1, 2 * i + ci, 2 * j + cj))
        else:
            tree.leaves.add(key)

    for j in range(layout[1]):
        for i in range(layout[0]):
            visit((0, i, j))
    return tree


def balance(tree: Tree, periodic):
    """2:1 grading across faces and corners, periodic seams included
    (`_balance!`, mesh.jl:673-714).  Splitting the coarser leaf of every
    violating pair until none remains reaches the unique minimal balanced
    refinement, which is what the reference's restart loop also produces."""
    layout = tree.layout
    changed = True
    while changed:
        changed = False
        for leaf in sorted(tree.leaves):
            if leaf not in tree.leaves:
                continue
            level, i, j = leaf
            if level < 2:
                continue
            nxl, nyl = layout[0] << level, layout[1] << level
            for dj in (-1, 0, 1):
                for di in (-1, 0, 1):
                    if di == 0 and dj == 0:
                        continue
                    ni, nj = i + di, j + dj
                    if periodic[0]:
                        ni %= nxl
                    elif not 0 <= ni < nxl:
                        continue
                    if periodic[1]:
                        nj %= nyl
                    elif not 0 <= nj < nyl:
                        continue
                    cover = tree.leaf_at(level, ni, nj)
                    if cover is not None and cover[0] + 1 < level:
                        tree.split(cover)
                        changed = True
    return tree


@dataclass
class Mesh:
    """Serial 2-D forest of fixed-size leaf blocks (mesh.jl:226-246)."""

    base_mesh: tuple
    block_size: tuple
    origin: tuple
    extent: tuple
    periodic: tuple
    max_level: int
    tree: Tree
    keys: list            # sorted leaf keys (level, i, j)
    block_origin: np.ndarray
    block_extent: np.ndarray
    spacing: np.ndarray   # (nblocks, 2)
    volume: np.ndarray    # (nblocks,)
    # interior faces (axis-major)
    face_minus: np.ndarray
    face_plus: np.ndarray
    face_axis: np.ndarray   # 1 or 2, as in the reference
    face_area: np.ndarray
    face_center: np.ndarray
    # boundary faces
    bface_cell: np.ndarray
    bface_axis: np.ndarray
    bface_side: np.ndarray
    bface_area: np.ndarray
    bface_center: np.ndarray
    key_index: dict = field(default_factory=dict)

    @property
    def nblocks(self):
        return len(self.keys)

    @property
    def ncells(self):
        return self.nblocks * self.block_size[0] * self.block_size[1]

    @property
    def nfaces(self):
        return len(self.face_minus)

    @property
    def active_level(self):
        return max(k[0] for k in self.keys)

    def lattice_size(self, level=None):
        """`_cells_at_level` (mesh.jl:436-437) at `level` (default: finest active)."""
        level = self.active_level if level is None else level
        return (self.base_mesh[0] << level, self.base_mesh[1] << level)

    def cell_lattice_bounds(self, cells, lattice):
        """`_cell_lattice_bounds` (mesh.jl:450-459), vectorised over cell indices."""
        nx, ny = self.block_size
        cells = np.asarray(cells)
        b = cells // (nx * ny)
        r = cells % (nx * ny)
        i = r % nx
        j = r // nx
        lev = self._key_level[b]
        sx = lattice[0] // (self.base_mesh[0] << lev)
        sy = lattice[1] // (self.base_mesh[1] << lev)
        lowx = (self._key_i[b] * nx + i) * sx
        lowy = (self._key_j[b] * ny + j) * sy
        return lowx, lowy, sx, sy

    def face_lattice_geometry(self, lattice):
        """`_face_lattice_geometry` (mesh.jl:461-474) for every interior face:
        (normal, lo, hi) on `lattice`, normal wrapped on periodic axes."""
        mlx, mly, msx, msy = self.cell_lattice_bounds(self.face_minus, lattice)
        plx, ply, psx, psy = self.cell_lattice_bounds(self.face_plus, lattice)
        ax = self.face_axis
        normal = np.where(ax == 1, mlx + msx, mly + msy)
        for a in (0, 1):
            if self.periodic[a]:
                sel = ax == a + 1
                normal[sel] = normal[sel] % lattice[a]
        lo = np.where(ax == 1, np.maximum(mly, ply), np.maximum(mlx, plx))
        hi = np.where(ax == 1, np.minimum(mly + msy, ply + psy), np.minimum(mlx + msx, plx + psx))
        return normal, lo, hi

    def bface_lattice_geometry(self, lattice):
        """Boundary-face form of `_face_lattice_geometry` (mesh.jl:476-485)."""
        lx, ly, sx, sy = self.cell_lattice_bounds(self.bface_cell, lattice)
        ax = self.bface_axis
        side = self.bface_side
        normal = np.where(ax == 1, lx + np.where(side > 0, sx, 0), ly + np.where(side > 0, sy, 0))
        lo = np.where(ax == 1, ly, lx)
        hi = np.where(ax == 1, ly + sy, lx + sx)
        return normal, lo, hi

    def cell_volumes(self):
        nx, ny = self.block_size
        return np.repeat(self.volume, nx * ny)

    def cell_centers(self):
        """`cellcenter` (mesh.jl:1136-1144) for every cell, in cell order."""
        nx, ny = self.block_size
        ii = np.tile(np.arange(nx), ny)
        jj = np.repeat(np.arange(ny), nx)
        x = self.block_origin[:, 0:1] + (ii[None, :] + 0.5) * self.spacing[:, 0:1]
        y = self.block_origin[:, 1:2] + (jj[None, :] + 0.5) * self.spacing[:, 1:2]
        return x.ravel(), y.ravel()


def _match_axis(mesh_keys, block_size, base_mesh, max_level, axis, periodic, origin, extent, lattice):
    """`_lattice_sides` + `_match_sides!` (mesh.jl:787-927) for one axis."""
    nx, ny = block_size
    lines = lattice[axis]
    t_axis = 1 - axis
    nb = len(mesh_keys)
    lev = np.array([k[0] for k in mesh_keys], dtype=np.int64)
    ki = np.array([k[1] for k in mesh_keys], dtype=np.int64)
    kj = np.array([k[2] for k in mesh_keys], dtype=np.int64)
    scale = (1 << (max_level - lev))
    ii = np.tile(np.arange(nx), ny)
    jj = np.repeat(np.arange(ny), nx)
    xlo = (ki[:, None] * nx * scale[:, None] + ii[None, :] * scale[:, None]).ravel()
    ylo = (kj[:, None] * ny * scale[:, None] + jj[None, :] * scale[:, None]).ravel()
    sc = np.repeat(scale, nx * ny)
    cell = np.arange(nb * nx * ny)
    if axis == 0:
        low, high, tlo, thi = xlo, xlo + sc, ylo, ylo + sc
    else:
        low, high, tlo, thi = ylo, ylo + sc, xlo, xlo + sc
    lower_line = high % lines if periodic else high
    upper_line = low % lines if periodic else low
    # stable grouping by line, then by `lo` (unique per side of a line)
    lower_order = np.lexsort((tlo, lower_line))
    upper_order = np.lexsort((tlo, upper_line))
    lower_counts = np.bincount(lower_line, minlength=lines + 1)
    upper_counts = np.bincount(upper_line, minlength=lines + 1)
    lower_off = np.concatenate(([0], np.cumsum(lower_counts)))
    upper_off = np.concatenate(([0], np.cumsum(upper_counts)))
    normal_scale = extent[axis] / lattice[axis]
    tangent_scale = extent[t_axis] / lattice[t_axis]
    fm, fp, fa, fc = [], [], [], []
    bc, bs, ba, bcen = [], [], [], []
    L_tlo = tlo[lower_order]; L_thi = thi[lower_order]; L_cell = cell[lower_order]
    U_tlo = tlo[upper_order]; U_thi = thi[upper_order]; U_cell = cell[upper_order]
    for line in range(lines + 1):
        li, lstop = lower_off[line], lower_off[line + 1]
        ui, ustop = upper_off[line], upper_off[line + 1]
        while li < lstop and ui < ustop:
            lo = max(L_tlo[li], U_tlo[ui])
            hi = min(L_thi[li], U_thi[ui])
            if lo < hi:
                normal = origin[axis] + line * normal_scale
                tangent = origin[t_axis] + (lo + hi) * tangent_scale / 2
                fm.append(L_cell[li]); fp.append(U_cell[ui])
                fa.append((hi - lo) * tangent_scale)
                fc.append((normal, tangent) if axis == 0 else (tangent, normal))
            lh, uh = L_thi[li], U_thi[ui]
            if lh <= uh:
                li += 1
            if uh <= lh:
                ui += 1
        for side_list, start, stop, side in ((0, li, lstop, 1), (1, ui, ustop, -1)):
            for k in range(start, stop):
                if side_list == 0:
                    rlo, rhi, c = L_tlo[k], L_thi[k], L_cell[k]
                else:
                    rlo, rhi, c = U_tlo[k], U_thi[k], U_cell[k]
                normal = origin[axis] + line * extent[axis] / lattice[axis]
                tangent = origin[t_axis] + (rlo + rhi) * extent[t_axis] / (2 * lattice[t_axis])
                bc.append(c); bs.append(side)
                ba.append((rhi - rlo) * extent[t_axis] / lattice[t_axis])
                bcen.append((normal, tangent) if axis == 0 else (tangent, normal))
    return fm, fp, fa, fc, bc, bs, ba, bcen


def mesh_from_tree(tree: Tree, base_mesh, block_size, periodic, max_level) -> Mesh:
    """`_leaf_blocks` + `_build_face_schedules` (mesh.jl:759-773, 874-895)."""
    keys = sorted(tree.leaves, key=lambda k: (k[0], k[2], k[1]))
    nb = len(keys)
    bo = np.zeros((nb, 2)); be = np.zeros((nb, 2))
    for b, key in enumerate(keys):
        o, e = tree.node_box(key)
        bo[b] = o; be[b] = e
    spacing = np.stack([be[:, 0] / block_size[0], be[:, 1] / block_size[1]], axis=1)
    volume = spacing[:, 0] * spacing[:, 1]
    active = max(k[0] for k in keys)
    lattice = (base_mesh[0] << active, base_mesh[1] << active)
    parts = [_match_axis(keys, block_size, base_mesh, active, a, periodic[a],
                         tree.origin, tree.extent, lattice) for a in (0, 1)]
    fm = np.array(parts[0][0] + parts[1][0], dtype=np.int64)
    fp = np.array(parts[0][1] + parts[1][1], dtype=np.int64)
    fax = np.array([1] * len(parts[0][0]) + [2] * len(parts[1][0]), dtype=np.int64)
    fa = np.array(parts[0][2] + parts[1][2], dtype=np.float64)
    fc = np.array(parts[0][3] + parts[1][3], dtype=np.float64).reshape(-1, 2)
    bcell = np.array(parts[0][4] + parts[1][4], dtype=np.int64)
    bax = np.array([1] * len(parts[0][4]) + [2] * len(parts[1][4]), dtype=np.int64)
    bside = np.array(parts[0][5] + parts[1][5], dtype=np.int64)
    barea = np.array(parts[0][6] + parts[1][6], dtype=np.float64)
    bcen = np.array(parts[0][7] + parts[1][7], dtype=np.float64).reshape(-1, 2)
    mesh = Mesh(tuple(base_mesh), tuple(block_size), tree.origin, tree.extent, tuple(periodic),
                max_level, tree, keys, bo, be, spacing, volume,
                fm, fp, fax, fa, fc, bcell, bax, bside, barea, bcen)
    mesh.key_index = {k: b for b, k in enumerate(keys)}
    mesh._key_level = np.array([k[0] for k in keys], dtype=np.int64)
    mesh._key_i = np.array([k[1] for k in keys], dtype=np.int64)
    mesh._key_j = np.array([k[2] for k in keys], dtype=np.int64)
    return mesh


def block_tree_mesh(*, block_size=(16, 16), base_mesh=None, origin=(0.0, 0.0), extent=(1.0, 1.0),
                    periodic=(True, True), max_level=0, refine=None, leaves=None) -> Mesh:
    """`BlockTreeMesh(; ...)` (mesh.jl:1059-1121).  Either a `refine(key, origin,
    extent)` callback (the reference's) or an explicit set of leaf `keys`."""
    base_mesh = tuple(block_size) if base_mesh is None else tuple(base_mesh)
    nx, ny = block_size
    if nx < 2 or ny < 2 or nx % 2 or ny % 2:
        raise ValueError("block dimensions must be even and at least two")
    if base_mesh[0] % nx or base_mesh[1] % ny or base_mesh[0] < nx or base_mesh[1] < ny:
        raise ValueError("base mesh dimensions must be integer multiples of block dimensions")
    if leaves is None:
        refine = refine or (lambda key, o, e: False)
        tree = build_tree(base_mesh, block_size, origin, extent, max_level, refine)
    else:
        layout = (base_mesh[0] // nx, base_mesh[1] // ny)
        tree = Tree(layout, tuple(map(float, origin)), tuple(map(float, extent)),
                    (extent[0] / layout[0], extent[1] / layout[1]))
        for key in leaves:
            key = tuple(int(v) for v in key)
            tree.leaves.add(key)
            lev, i, j = key
            for l in range(lev):
                tree.internal.add((l, i >> (lev - l), j >> (lev - l)))
        tree.leaves -= tree.internal
    balance(tree, periodic)
    return mesh_from_tree(tree, base_mesh, block_size, periodic, max_level)
