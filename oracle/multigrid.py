"""Oracle (test infrastructure only): CPU restatement of TwoPhaseAMR.jl's
rediscretized tree geometric multigrid preconditioner and its V-cycle.

Reference (ronaldremmerswaal/TwoPhaseAMR.jl):
  src/solvers/multigrid/tree_coarsening.jl:30-57    `_all_leaf_pruned_mesh`
  src/solvers/multigrid/tree_coarsening.jl:62-82    `_coarsened_base_mesh`
  src/solvers/multigrid/tree_coarsening.jl:169-212  stopping rules, `_tree_next_coarse_mesh!`
  src/solvers/multigrid/tree_coarsening.jl:228-252  `_tree_cell_prolongation` (owners)
  src/solvers/multigrid/tree_coarsening.jl:335-398  `_face_coefficient_restriction`
  src/solvers/multigrid/tree_coarsening.jl:538-555  `_restrict_face_coefficients!`
  src/solvers/multigrid/hierarchy.jl:8-30           `_jacobi_weight!`
  src/solvers/multigrid/hierarchy.jl:208-246        `_prolongate!`, `_restrict!`
  src/solvers/multigrid/hierarchy.jl:316-343        component projections
  src/solvers/multigrid/hierarchy.jl:631-721        `_smoothed_transfer_refresh`
  src/solvers/multigrid/hierarchy.jl:786-817        `_multigrid_level`
  src/solvers/multigrid/geometric_preconditioner.jl:144-169, 171-442  hierarchy build
  src/solvers/multigrid/cycles.jl:8-77              `_smooth!`, `_coarse_solve!`, `_vcycle!`
  src/solvers/multigrid/cycles.jl:262-283           `ldiv!`

The coarse factorization is SciPy's SuperLU in place of UMFPACK (any exact
factorization agrees to rounding).
"""
from __future__ import annotations

import bisect
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .mesh import Tree, balance, mesh_from_tree
from .operator import PoissonOperator


@dataclass
class MultigridOptions:
    """`MultigridOptions` (src/solvers/multigrid/options.jl:14-48)."""

    coarse_size: int = 64
    pre_sweeps: int = 2
    post_sweeps: int = 2
    max_levels: int = 32
    # not in the reference: "red_black" replaces its damped Jacobi sweeps by
    # red-black Gauss-Seidel (see `red_black_colours`)
    smoother: str = "jacobi"

    def __post_init__(self):
        for v in (self.coarse_size, self.pre_sweeps, self.post_sweeps, self.max_levels):
            if not isinstance(v, (int, np.integer)) or isinstance(v, bool):
                raise TypeError("multigrid sizes and sweep counts must be integers")
        if self.smoother not in ("jacobi", "red_black"):
            raise ValueError("smoother must be 'jacobi' or 'red_black'")
        if self.coarse_size <= 0:
            raise ValueError("coarse_size must be positive")
        if self.pre_sweeps < 0 or self.post_sweeps < 0:
            raise ValueError("sweep counts must be nonnegative")
        if self.max_levels <= 0:
            raise ValueError("max_levels must be positive")


def all_leaf_pruned_mesh(mesh):
    """Replace every terminal sibling family by its parent, then rebalance
    (tree_coarsening.jl:30-57)."""
    old = mesh.tree
    internal = {n for n in old.internal
                if any((n[0] + 1, 2 * n[1] + ci, 2 * n[2] + cj) in old.internal
                       for ci in (0, 1) for cj in (0, 1))}
    tree = Tree(old.layout, old.origin, old.extent, old.root_extent)
    tree.internal = set(internal)
    for j in range(old.layout[1]):
        for i in range(old.layout[0]):
            if (0, i, j) not in internal:
                tree.leaves.add((0, i, j))
    for n in internal:
        for cj in (0, 1):
            for ci in (0, 1):
                c = (n[0] + 1, 2 * n[1] + ci, 2 * n[2] + cj)
                if c not in internal:
                    tree.leaves.add(c)
    balance(tree, mesh.periodic)
    max_level = max(k[0] for k in internal) + 1 if internal else 0
    return mesh_from_tree(tree, mesh.base_mesh, mesh.block_size, mesh.periodic, max_level)


def coarsened_base_mesh(mesh):
    """Agglomerate 2x2 roots (tree_coarsening.jl:62-82); None when impossible."""
    layout = mesh.tree.layout
    if layout[0] % 2 or layout[1] % 2:
        return None
    base = (mesh.base_mesh[0] // 2, mesh.base_mesh[1] // 2)
    for a in (0, 1):
        if mesh.periodic[a] and base[a] < 4:
            return None
    nl = (base[0] // mesh.block_size[0], base[1] // mesh.block_size[1])
    tree = Tree(nl, mesh.origin, mesh.extent, (mesh.extent[0] / nl[0], mesh.extent[1] / nl[1]))
    tree.leaves = {(0, i, j) for j in range(nl[1]) for i in range(nl[0])}
    return mesh_from_tree(tree, base, mesh.block_size, mesh.periodic, 0)


def next_coarse_mesh(current, coarse_size, max_levels, number_of_levels):
    """`_tree_next_coarse_mesh!` with pruning=:all (tree_coarsening.jl:187-212)."""
    if not (current.ncells > coarse_size and number_of_levels < max_levels):
        return None
    coarse = coarsened_base_mesh(current) if current.active_level == 0 else all_leaf_pruned_mesh(current)
    if coarse is None or coarse.ncells >= current.ncells:
        return None
    return coarse


def common_lattice(fine, coarse):
    """`_tree_common_lattice_size` (tree_coarsening.jl:335-339), at active levels."""
    a = fine.lattice_size(); b = coarse.lattice_size()
    return (max(a[0], b[0]), max(a[1], b[1]))


def cell_owners(fine, coarse):
    """`_tree_cell_prolongation` (tree_coarsening.jl:228-252): the coarse cell that
    contains each fine cell (lattice point low + scale/2)."""
    lattice = common_lattice(fine, coarse)
    lx, ly, sx, sy = fine.cell_lattice_bounds(np.arange(fine.ncells), lattice)
    px = lx + sx // 2
    py = ly + sy // 2
    nx, ny = coarse.block_size
    tree = coarse.tree
    root_w = (lattice[0] // tree.layout[0], lattice[1] // tree.layout[1])
    owners = np.empty(fine.ncells, dtype=np.int64)
    for c in range(fine.ncells):
        x, y = int(px[c]), int(py[c])
        i, j = x // root_w[0], y // root_w[1]
        key = (0, i, j)
        while key not in tree.leaves:
            level = key[0] + 1
            cw = (root_w[0] >> level, root_w[1] >> level)
            key = (level, x // cw[0], y // cw[1])
        level = key[0]
        scale = (lattice[0] // ((tree.layout[0] * nx) << level),
                 lattice[1] // ((tree.layout[1] * ny) << level))
        ci = (x // scale[0]) % nx
        cj = (y // scale[1]) % ny
        owners[c] = coarse.key_index[key] * nx * ny + cj * nx + ci
    return owners


def face_coefficient_restriction(coarse, fine, boundary=False):
    """`_face_coefficient_restriction` (tree_coarsening.jl:347-398): CSR rows of
    coarse faces over fine faces on the same lattice line, weighted by overlap;
    with `boundary`, the same over the boundary faces."""
    lattice = common_lattice(fine, coarse)
    if boundary:
        fn, flo, fhi = fine.bface_lattice_geometry(lattice)
        faxis, nfine = fine.bface_axis, len(fine.bface_cell)
        cgeo, caxis, ncoarse = coarse.bface_lattice_geometry(lattice), coarse.bface_axis, len(coarse.bface_cell)
    else:
        fn, flo, fhi = fine.face_lattice_geometry(lattice)
        faxis, nfine = fine.face_axis, fine.nfaces
        cgeo, caxis, ncoarse = coarse.face_lattice_geometry(lattice), coarse.face_axis, coarse.nfaces
    lines = {}
    for f in range(nfine):
        lines.setdefault((int(faxis[f]), int(fn[f])), []).append((int(flo[f]), int(fhi[f]), f))
    starts = {}
    for key, v in lines.items():
        v.sort(key=lambda t: t[0])
        starts[key] = [t[0] for t in v]
    cn, clo, chi = cgeo
    ptr = [0]; idx = []; w = []
    for f in range(ncoarse):
        lo, hi = int(clo[f]), int(chi[f])
        covered = 0
        key = (int(caxis[f]), int(cn[f]))
        line = lines.get(key, [])
        # fine faces on a line are disjoint and sorted: start at the one that
        # contains lo (the scan order, and so the sums, are unchanged)
        first = max(bisect.bisect_right(starts[key], lo) - 1, 0) if line else 0
        for (a, b, k) in line[first:]:
            if a >= hi:
                break
            overlap = min(hi, b) - max(lo, a)
            if overlap > 0:
                idx.append(k); w.append(overlap / (hi - lo)); covered += overlap
        if covered != hi - lo:
            raise RuntimeError("tree hierarchy could not cover a coarse face with fine faces")
        ptr.append(len(idx))
    return sp.csr_matrix((np.array(w), np.array(idx, dtype=np.int64), np.array(ptr)),
                         shape=(ncoarse, nfine))


def jacobi_weight(diagonal, row_sums, *, skip_nonpositive=False, allow_zero=False,
                  clamp=True, zero_weight=1.0):
    """`_jacobi_weight!` (hierarchy.jl:8-30): returns (inverse diagonal, weight)."""
    inv = diagonal.astype(np.float64).copy()
    bound = 0.0
    for k in range(len(inv)):
        d = inv[k]
        if d == 0 and allow_zero:
            continue
        if not d > 0:
            if skip_nonpositive:
                continue
            raise ValueError("elliptic matrix has a non-positive diagonal")
        bound = max(bound, row_sums[k] / d)
        inv[k] = 1.0 / d
    if bound == 0:
        return inv, zero_weight
    weight = 4.0 / (3.0 * bound)
    return inv, (min(1.0, weight) if clamp else weight)


def smoothed_transfer(stiffness, owners, n_coarse):
    """`P = (I - w D^-1 A) P_tent` with an unclamped weight
    (`_smoothed_transfer_refresh`, hierarchy.jl:631-721)."""
    n = stiffness.shape[0]
    d = stiffness.diagonal()
    rs = np.asarray(abs(stiffness).sum(axis=1)).ravel()
    inv, w = jacobi_weight(d, rs, skip_nonpositive=True, clamp=False, zero_weight=0.0)
    Pt = sp.csr_matrix((np.ones(n), (np.arange(n), owners)), shape=(n, n_coarse))
    P = (Pt - sp.diags(w * inv) @ stiffness @ Pt).tocsr()
    P.sort_indices()
    return P, w


def red_black_colours(mesh):
    """Red-black colouring of a level (no counterpart in the reference, which
    smooths with damped Jacobi): colour (I + J) mod 2 of every cell, with (I, J)
    its lattice coordinates at its own block's refinement level (0 red, 1 black)."""
    nx, ny = mesh.block_size
    ci = np.tile(np.arange(nx), ny)
    cj = np.repeat(np.arange(ny), nx)
    out = np.empty(mesh.ncells, dtype=np.int64)
    for b, (_, bi, bj) in enumerate(mesh.keys):
        out[b * nx * ny:(b + 1) * nx * ny] = (bi * nx + ci + bj * ny + cj) & 1
    return out


def red_black_weight(matrix, colours):
    """Weight of a red-black half-sweep: `_jacobi_weight!`'s rule min(1, 4/(3 b))
    applied to the rows restricted to their own colour, b = max_i sum over j of
    the same colour of |a_ij| / a_ii (1, so weight 1, for an exact two-colouring;
    above 1 where coarse-fine faces, hanging-vertex rows or odd periodic axes
    couple cells of one colour)."""
    A = matrix.tocoo()
    same = colours[A.row] == colours[A.col]
    rs = np.zeros(matrix.shape[0])
    np.add.at(rs, A.row[same], np.abs(A.data[same]))
    d = matrix.diagonal()
    ok = d > 0
    bound = float(np.max(rs[ok] / d[ok])) if np.any(ok) else 0.0
    return 1.0 if bound == 0.0 else min(1.0, 4.0 / (3.0 * bound))


class Level:
    """`MultigridLevel` (hierarchy.jl:248-274) built by `_multigrid_level`."""

    def __init__(self, op: PoissonOperator, prolongation=None):
        self.op = op
        self.matrix = op.matrix
        self.volumes = op.volumes
        d = op.matrix.diagonal()
        rs = np.asarray(abs(op.matrix).sum(axis=1)).ravel()
        self.inverse_diagonal, self.weight = jacobi_weight(d, rs, allow_zero=op.singular)
        self.prolongation = prolongation
        comp = op.components
        self.slots = comp["slots"]
        self.component_volumes = comp["volumes"] if op.singular else np.zeros(0)
        self.n = op.mesh.ncells
        self.colours = red_black_colours(op.mesh)
        self.rb_weight = red_black_weight(op.matrix, self.colours)

    @property
    def singular(self):
        return len(self.component_volumes) > 0

    def project_rhs(self, b):
        """`_multigrid_project_component_rhs!` (hierarchy.jl:330-343)."""
        for s, cv in enumerate(self.component_volumes):
            sel = self.slots == s
            b[sel] -= self.volumes[sel] * (np.sum(b[sel]) / cv)
        return b

    def remove_means(self, x):
        """`_multigrid_remove_component_means!` (hierarchy.jl:316-328)."""
        for s, cv in enumerate(self.component_volumes):
            sel = self.slots == s
            x[sel] -= np.sum(self.volumes[sel] * x[sel]) / cv
        return x


class TreeGeometricMultigrid:
    """`TreeGeometricMultigridPreconditioner` (geometric_preconditioner.jl:50-442)."""

    def __init__(self, op: PoissonOperator, options: MultigridOptions = None):
        options = options or MultigridOptions()
        self.options = options
        self.pre_sweeps, self.post_sweeps = options.pre_sweeps, options.post_sweeps
        ops = [op]
        self.owners = []
        self.prolongations = []
        self.transfer_weights = []
        self.restrictions = []
        self.boundary_restrictions = []
        current = op.mesh
        while True:
            coarse = next_coarse_mesh(current, options.coarse_size, options.max_levels, len(ops))
            if coarse is None:
                break
            owners = cell_owners(current, coarse)
            P, w = smoothed_transfer(ops[-1].matrix, owners, coarse.ncells)
            R = face_coefficient_restriction(coarse, current)
            kappa_c = R @ ops[-1].face_coefficient
            self.owners.append(owners)
            self.prolongations.append(P)
            self.transfer_weights.append(w)
            self.restrictions.append(R)
            # open sides keep their Dirichlet conductance on every level: the
            # boundary coefficients are restricted like the interior ones
            # (geometric_preconditioner.jl:256-300)
            kb_c = None
            if any(op.open_sides):
                Rb = face_coefficient_restriction(coarse, current, boundary=True)
                self.boundary_restrictions.append(Rb)
                kb_c = Rb @ ops[-1].boundary_coefficient
            ops.append(PoissonOperator(coarse, kappa_c, open_sides=op.open_sides, boundary_coefficient=kb_c))
            current = coarse
        self.operators = ops
        self.levels = [Level(o, self.prolongations[k] if k < len(self.prolongations) else None)
                       for k, o in enumerate(ops)]
        self._factor_coarse()

    def _factor_coarse(self):
        """`_augmented_multigrid_coarse_matrix` + LU (geometric_preconditioner.jl:144-169, 420-430)."""
        c = self.levels[-1]
        n = c.n
        if c.singular:
            nc = len(c.component_volumes)
            rows = np.arange(n)[c.slots >= 0]
            C = sp.csr_matrix((c.volumes[rows], (rows, c.slots[rows])), shape=(n, nc))
            A = sp.bmat([[c.matrix, C], [C.T, None]]).tocsc()
        else:
            A = c.matrix.tocsc()
        self.coarse_matrix = A
        self.coarse_lu = spla.splu(A)

    def refresh(self, kappa):
        """`_refresh_geometric_multigrid!` (geometric_preconditioner.jl:483-594)."""
        self.operators[0].refresh(kappa)
        for k in range(1, len(self.operators)):
            if self.boundary_restrictions:
                # the fine level's (possibly updated) open-face coefficients,
                # restricted again (geometric_preconditioner.jl:505-515)
                self.operators[k].update_boundary_coefficient(
                    self.boundary_restrictions[k - 1] @ self.operators[k - 1].boundary_coefficient)
            self.operators[k].refresh(self.restrictions[k - 1] @ self.operators[k - 1].face_coefficient)
        for k in range(len(self.prolongations)):
            P, w = smoothed_transfer(self.operators[k].matrix, self.owners[k], self.operators[k + 1].mesh.ncells)
            self.prolongations[k] = P
            self.transfer_weights[k] = w
        self.levels = [Level(o, self.prolongations[k] if k < len(self.prolongations) else None)
                       for k, o in enumerate(self.operators)]
        self._factor_coarse()
        return self

    def coarse_solve(self, b):
        c = self.levels[-1]
        if c.singular:
            rhs = np.zeros(self.coarse_matrix.shape[0])
            rhs[:c.n] = b
            return self.coarse_lu.solve(rhs)[:c.n]
        return self.coarse_lu.solve(b)

    def smooth(self, lev: Level, x, b, sweeps, order=(0, 1)):
        """`_smooth!` (cycles.jl:8-24): damped Jacobi, means removed per sweep.
        With the red-black smoother each sweep updates the colours in `order`
        (red then black before the coarse correction, the reverse after it, so
        that the V-cycle stays symmetric), each colour from the iterate left by
        the previous one, with `red_black_weight`."""
        for _ in range(sweeps):
            if self.options.smoother == "red_black":
                om = lev.rb_weight
                for c in order:
                    t = lev.matrix @ x
                    sel = lev.colours == c
                    x[sel] += om * lev.inverse_diagonal[sel] * (b[sel] - t[sel])
            else:
                t = lev.matrix @ x
                x += lev.weight * lev.inverse_diagonal * (b - t)
            if lev.singular:
                lev.remove_means(x)
        return x

    def vcycle(self, k, b):
        """`_vcycle!` (cycles.jl:46-77); returns the level-k correction."""
        lev = self.levels[k]
        if lev.singular:
            lev.project_rhs(b)
        if k == len(self.levels) - 1:
            return self.coarse_solve(b)
        x = np.zeros(lev.n)
        self.smooth(lev, x, b, self.pre_sweeps)
        r = b - lev.matrix @ x
        bc = lev.prolongation.T @ r + 0.0
        xc = self.vcycle(k + 1, bc)
        x += lev.prolongation @ xc
        if lev.singular:
            lev.remove_means(x)
        self.smooth(lev, x, b, self.post_sweeps, order=(1, 0))
        return x

    def ldiv(self, r):
        """`ldiv!(z, P, r)` (cycles.jl:262-283)."""
        return self.vcycle(0, np.array(r, dtype=np.float64, copy=True))

    @property
    def level_sizes(self):
        return [lev.n for lev in self.levels]
