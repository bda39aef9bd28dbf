"""`BlockTreeMesh`: the block quadtree forest the pressure solve runs on.

Mirrors `BlockTreeMesh(; base_mesh, block_size, origin, extent, periodic,
max_level, refine)` (src/mesh/topology/mesh.jl:1059-1121 in
ronaldremmerswaal/TwoPhaseAMR.jl).  The `refine(key, origin, extent)` callback
is evaluated here, on the host, exactly as `_build_tree` does (mesh.jl:716-734);
the library then restores 2:1 grading, orders the blocks by (level, j, i) and
builds the face schedules (mesh.jl:673-937).  Indices are 0-based.
"""
from __future__ import annotations

from collections import namedtuple

import numpy as np

from . import _lib

BlockKey = namedtuple("BlockKey", "level i j")


def _leaves(base_mesh, block_size, origin, extent, max_level, refine):
    layout = (base_mesh[0] // block_size[0], base_mesh[1] // block_size[1])
    root_extent = (extent[0] / layout[0], extent[1] / layout[1])
    out = []

    def visit(key, o, e):
        if key.level >= max_level or not refine(key, o, e):
            out.append(key)
            return
        he = (e[0] / 2, e[1] / 2)
        for cj in (0, 1):
            for ci in (0, 1):
                child = BlockKey(key.level + 1, 2 * key.i + ci, 2 * key.j + cj)
                visit(child, (o[0] + he[0] if ci else o[0], o[1] + he[1] if cj else o[1]), he)

    for j in range(layout[1]):
        for i in range(layout[0]):
            visit(BlockKey(0, i, j), (origin[0] + i * root_extent[0], origin[1] + j * root_extent[1]), root_extent)
    return out


class BlockTreeMesh:
    """Serial 2-D forest of fixed-size Cartesian leaf blocks."""

    def __init__(self, *, block_size=(16, 16), base_mesh=None, origin=(0.0, 0.0), extent=(1.0, 1.0),
                 periodic=(True, True), max_level=0, refine=None, leaves=None):
        base_mesh = tuple(block_size) if base_mesh is None else tuple(base_mesh)
        for v in base_mesh:
            if not isinstance(v, (int, np.integer)) or isinstance(v, bool):
                raise TypeError("base mesh dimensions must be integers")
        if max_level < 0:
            raise ValueError("max_level must be nonnegative")
        self.base_mesh = tuple(int(v) for v in base_mesh)
        self.block_size = tuple(int(v) for v in block_size)
        self.origin = tuple(float(v) for v in origin)
        self.extent = tuple(float(v) for v in extent)
        self.periodic = tuple(bool(v) for v in periodic)
        self.max_level = int(max_level)
        if leaves is None:
            if self.block_size[0] < 2 or self.block_size[1] < 2:
                raise ValueError("block dimensions must be at least two")
            if self.block_size[0] % 2 or self.block_size[1] % 2:
                raise ValueError("block dimensions must be even for dyadic transfer")
            if any(b % s for b, s in zip(self.base_mesh, self.block_size)):
                raise ValueError("base mesh dimensions must be integer multiples of block dimensions")
            refine = refine or (lambda key, o, e: False)
            leaves = _leaves(self.base_mesh, self.block_size, self.origin, self.extent, self.max_level, refine)
        self._leaf_keys = np.ascontiguousarray(np.array([tuple(k) for k in leaves], dtype=np.int32).reshape(-1, 3))
        self.ctx = _lib.Context(0)
        self.ctx.call("tpa_set_mesh", *self._mesh_args())
        sizes = np.zeros(5, dtype=np.int64)
        self.ctx.call("tpa_mesh_sizes", _lib.ptr(sizes, _lib.C.c_int64))
        self.nblocks, self.ncells, self.nfaces, self.nboundary_faces, self.finest_level = (int(v) for v in sizes)
        keys = np.zeros((self.nblocks, 3), dtype=np.int32)
        geom = np.zeros((self.nblocks, 5), dtype=np.float64)
        self.ctx.call("tpa_mesh_blocks", _lib.ptr(keys, _lib.C.c_int32), _lib.ptr(geom, _lib.C.c_double))
        self.keys = keys
        self.block_origin = geom[:, 0:2].copy()
        self.spacing = geom[:, 2:4].copy()
        self.volume = geom[:, 4].copy()
        nf = self.nfaces
        self.face_minus = np.zeros(nf, dtype=np.int32)
        self.face_plus = np.zeros(nf, dtype=np.int32)
        self.face_axis = np.zeros(nf, dtype=np.int8)
        self.face_area = np.zeros(nf, dtype=np.float64)
        self.ctx.call("tpa_mesh_faces", _lib.ptr(self.face_minus, _lib.C.c_int32), _lib.ptr(self.face_plus, _lib.C.c_int32),
                      _lib.ptr(self.face_axis, _lib.C.c_int8), _lib.ptr(self.face_area, _lib.C.c_double))
        nb = self.nboundary_faces
        self.bface_cell = np.zeros(nb, dtype=np.int32)
        self.bface_axis = np.zeros(nb, dtype=np.int8)
        self.bface_side = np.zeros(nb, dtype=np.int8)
        self.bface_area = np.zeros(nb, dtype=np.float64)
        self.ctx.call("tpa_mesh_boundary_faces", _lib.ptr(self.bface_cell, _lib.C.c_int32),
                      _lib.ptr(self.bface_axis, _lib.C.c_int8), _lib.ptr(self.bface_side, _lib.C.c_int8),
                      _lib.ptr(self.bface_area, _lib.C.c_double))

    def _mesh_args(self):
        C = _lib.C
        self._args = (np.array(self.base_mesh, dtype=np.int32), np.array(self.block_size, dtype=np.int32),
                      np.array(self.periodic, dtype=np.int32), np.array(self.origin), np.array(self.extent))
        b, s, p, o, e = self._args
        return (_lib.ptr(b, C.c_int32), _lib.ptr(s, C.c_int32), _lib.ptr(p, C.c_int32), _lib.ptr(o, C.c_double),
                _lib.ptr(e, C.c_double), C.c_int64(len(self._leaf_keys)), _lib.ptr(self._leaf_keys, C.c_int32))

    @property
    def leaf_keys(self):
        return self._leaf_keys

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

    def face_centers(self):
        """Physical centre of every interior face (mesh.jl:897-927)."""
        xm, ym = self.cell_centers()
        nx, ny = self.block_size
        bm = self.face_minus // (nx * ny)
        bp = self.face_plus // (nx * ny)
        ax = self.face_axis
        cx = np.where(ax == 1, xm[self.face_minus] + self.spacing[bm, 0] / 2,
                      0.5 * (np.maximum(xm[self.face_minus] - self.spacing[bm, 0] / 2, xm[self.face_plus] - self.spacing[bp, 0] / 2)
                             + np.minimum(xm[self.face_minus] + self.spacing[bm, 0] / 2, xm[self.face_plus] + self.spacing[bp, 0] / 2)))
        cy = np.where(ax == 2, ym[self.face_minus] + self.spacing[bm, 1] / 2,
                      0.5 * (np.maximum(ym[self.face_minus] - self.spacing[bm, 1] / 2, ym[self.face_plus] - self.spacing[bp, 1] / 2)
                             + np.minimum(ym[self.face_minus] + self.spacing[bm, 1] / 2, ym[self.face_plus] + self.spacing[bp, 1] / 2)))
        if self.periodic[0]:
            cx = np.where((ax == 1) & (cx >= self.origin[0] + self.extent[0] - self.spacing[bm, 0] / 4), cx - self.extent[0], cx)
        if self.periodic[1]:
            cy = np.where((ax == 2) & (cy >= self.origin[1] + self.extent[1] - self.spacing[bm, 1] / 4), cy - self.extent[1], cy)
        return cx, cy
