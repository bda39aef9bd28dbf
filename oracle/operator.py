"""Oracle (test infrastructure only): CPU restatement of TwoPhaseAMR.jl's
cell-centred pressure operator `S = C' A sqrt(k) K sqrt(k) A C`.

Reference (ronaldremmerswaal/TwoPhaseAMR.jl):
  src/operators/elliptic.jl:157-257    `_integrated_stiffness` ((A+A')/2 of J'MJ)
  src/operators/elliptic.jl:520-545    `EllipticOperator` fields
  src/operators/elliptic.jl:683-800    constructor (zero reaction, unit diffusion)
  src/operators/elliptic.jl:969-980    `PoissonOperator`
  src/operators/elliptic.jl:1020-1042  `_cell_face_incidence`
  src/operators/elliptic.jl:1125-1180  `mul!` of `FactorizedEllipticOperator`
  src/operators/elliptic.jl:1272-1297  `weighted_gradient!`
  src/solvers/multigrid/elliptic_solver.jl:1-151  component labels, gauges and
                                        `_remove_component_volume_means!`
  src/two_phase/projection/common.jl:53-83  `_projection_component_labels!`
  src/operators/elliptic.jl:76-87      `_pressure_boundary_sides`, `_pressure_open_face`
  src/operators/elliptic.jl:91-134     `_boundary_material` (open-face coefficients
                                        extended from the opposite interior faces)
  src/operators/elliptic.jl:136-152    `_elliptic_boundary_data!` (open-face Dirichlet
                                        conductances: boundary diagonal and gradient)
  src/operators/elliptic.jl:1254-1262  `_elliptic_boundary_gradient!`

The configuration of the pressure projection is restated: reaction 0,
diffusion 1, no inactive cells; sides may be open (pressure Dirichlet 0:
Outflow / ZeroGradientVelocity), which adds 2 k_b / h |f| to the diagonal of
the cell at an open face and anchors its component.  Sparse sums are evaluated
by scipy, so assembled values agree with the reference to rounding, not
bitwise.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .metric import assemble_inverse_metric


def open_face_mask(mesh, open_sides):
    """`_pressure_open_face` (elliptic.jl:86-87) per boundary face; open_sides
    is (left, right, bottom, top) as `_pressure_boundary_sides`."""
    sides = tuple(bool(v) for v in (open_sides or (False,) * 4))
    ax, sd = mesh.bface_axis, mesh.bface_side
    idx = 2 * (ax.astype(np.int64) - 1) + (sd > 0)
    return np.array(sides)[idx] if len(ax) else np.zeros(0, dtype=bool)


def boundary_material(mesh, face_coefficient, open_sides):
    """`_boundary_material` (elliptic.jl:91-134) for a vector of interior
    coefficients: each open boundary face takes the area-weighted mean of the
    interior faces on the opposite side of its cell along its axis."""
    nb = len(mesh.bface_cell)
    values = np.zeros(nb)
    mask = open_face_mask(mesh, open_sides)
    if not mask.any():
        return values
    kappa = np.full(mesh.nfaces, float(face_coefficient)) if np.isscalar(face_coefficient) \
        else np.asarray(face_coefficient, dtype=np.float64)
    if np.isscalar(face_coefficient):
        values[mask] = float(face_coefficient)
        return values
    index = {(int(mesh.bface_cell[b]), int(mesh.bface_axis[b]), int(mesh.bface_side[b])): b
             for b in range(nb) if mask[b]}
    weights = np.zeros(nb)
    for f in range(mesh.nfaces):
        for cell, side in ((int(mesh.face_minus[f]), -1), (int(mesh.face_plus[f]), 1)):
            b = index.get((cell, int(mesh.face_axis[f]), side))
            if b is None:
                continue
            values[b] += mesh.face_area[f] * kappa[f]
            weights[b] += mesh.face_area[f]
    for b in np.flatnonzero(mask):
        if not weights[b] > 0:
            raise ValueError("cannot extend an interior coefficient to an open face without an opposite "
                             "interior face; supply boundary_face_coefficient")
        values[b] /= weights[b]
    return values


def boundary_data(mesh, material, open_sides, volumes):
    """`_elliptic_boundary_data!` (elliptic.jl:136-152) with unit apertures:
    the diagonal 2 k_b / h |f| per cell and the gradient factor 2 k_b / h per
    open boundary face (h: the cell's spacing along the face axis)."""
    nb = len(mesh.bface_cell)
    diagonal = np.zeros(mesh.ncells)
    gradient = np.zeros(nb)
    mask = open_face_mask(mesh, open_sides)
    nx, ny = mesh.block_size
    for b in np.flatnonzero(mask):
        cell = int(mesh.bface_cell[b])
        if not volumes[cell] > 0:
            continue
        ax = int(mesh.bface_axis[b]) - 1
        factor = 2 * material[b] / mesh.spacing[cell // (nx * ny), ax]
        gradient[b] = factor
        diagonal[cell] += mesh.bface_area[b] * factor
    return diagonal, gradient


class PoissonOperator:
    """`PoissonOperator(mesh; face_coefficient, velocity_boundary,
    boundary_face_coefficient)` (elliptic.jl:969-980, 683-800).  open_sides:
    (left, right, bottom, top) open (pressure Dirichlet) or None (closed);
    boundary_coefficient: one per boundary face, or None to extend the
    interior coefficients (`_boundary_material`)."""

    def __init__(self, mesh, face_coefficient=1.0, metric=None, open_sides=None, boundary_coefficient=None):
        self.mesh = mesh
        self.open_sides = tuple(bool(v) for v in (open_sides or (False,) * 4))
        nb = len(mesh.bface_cell)
        if boundary_coefficient is None:
            self.boundary_coefficient = boundary_material(mesh, face_coefficient, self.open_sides)
        else:
            bc = np.asarray(boundary_coefficient, dtype=np.float64).copy()
            if bc.shape != (nb,):
                raise ValueError("one coefficient is required per boundary face")
            if not np.all(np.isfinite(bc)) or np.any(bc < 0):
                raise ValueError("boundary coefficients must be finite and nonnegative")
            self.boundary_coefficient = bc
        nf, nc = mesh.nfaces, mesh.ncells
        kappa = np.full(nf, float(face_coefficient)) if np.isscalar(face_coefficient) \
            else np.asarray(face_coefficient, dtype=np.float64).copy()
        if kappa.shape != (nf,):
            raise ValueError("one coefficient is required per interior face")
        if not np.all(np.isfinite(kappa)) or np.any(kappa < 0):
            raise ValueError("face coefficients must be finite and nonnegative")
        self.face_coefficient = kappa
        self.sqrt_kappa = np.sqrt(kappa)
        if metric is None:
            metric = assemble_inverse_metric(mesh)
        self.K, self.diagonal_metric, self.metric_templates = metric
        self.volumes = mesh.cell_volumes()
        # area-weighted jump J: -|f| at the minus cell, +|f| at the plus cell
        f = np.arange(nf)
        self.J = sp.csr_matrix(
            (np.concatenate([-mesh.face_area, mesh.face_area]),
             (np.concatenate([f, f]), np.concatenate([mesh.face_minus, mesh.face_plus]))),
            shape=(nf, nc))
        self.boundary_diagonal, self.boundary_gradient = boundary_data(
            mesh, self.boundary_coefficient, self.open_sides, self.volumes)
        self.refresh(kappa)

    def weighted_metric(self):
        """`M = k K` (diagonal K) or `sqrt(k) K sqrt(k)` (elliptic.jl:185-195)."""
        if self.diagonal_metric:
            return sp.diags(self.face_coefficient * self.K.diagonal())
        s = sp.diags(self.sqrt_kappa)
        return (s @ self.K @ s).tocsc()

    def update_boundary_coefficient(self, material):
        """`_update_elliptic_boundary_coefficient!` (elliptic.jl:826-845): new
        open-face coefficients, boundary data and components; follow with
        `refresh` to re-assemble."""
        bc = np.asarray(material, dtype=np.float64).copy()
        if bc.shape != self.boundary_coefficient.shape:
            raise ValueError("one coefficient is required per boundary face")
        if not np.all(np.isfinite(bc)) or np.any(bc < 0):
            raise ValueError("boundary coefficients must be finite and nonnegative")
        self.boundary_coefficient = bc
        self.boundary_diagonal, self.boundary_gradient = boundary_data(
            self.mesh, bc, self.open_sides, self.volumes)
        return self

    def refresh(self, kappa):
        """`_update_elliptic_face_coefficient!` (elliptic.jl:847-916): new face
        coefficients on the fixed topology."""
        self.face_coefficient = np.asarray(kappa, dtype=np.float64).copy()
        self.sqrt_kappa = np.sqrt(self.face_coefficient)
        A = (self.J.T @ self.weighted_metric() @ self.J).tocsr()
        A = ((A + A.T) / 2).tocsr()
        if np.any(self.boundary_diagonal):
            A = (A + sp.diags(self.boundary_diagonal)).tocsr()
        A.sort_indices()
        self.matrix = A
        self.components = components(self)
        self.singular = len(self.components["anchors"]) > 0
        return self

    def apply(self, x):
        """Factorized action `mul!` (elliptic.jl:1125-1180)."""
        face_input = self.sqrt_kappa * (self.J @ x)
        face_output = self.K @ face_input
        return self.boundary_diagonal * x + self.J.T @ (self.sqrt_kappa * face_output)

    def weighted_gradient(self, p):
        """`weighted_gradient!` interior values (elliptic.jl:1272-1297)."""
        jump = self.mesh.face_area * (p[self.mesh.face_plus] - p[self.mesh.face_minus])
        return self.sqrt_kappa * (self.K @ (self.sqrt_kappa * jump))

    def boundary_weighted_gradient(self, p):
        """`_elliptic_boundary_gradient!` (elliptic.jl:1254-1262): -side k_b
        2/h p_cell on open faces, zero on closed ones."""
        return -self.mesh.bface_side * self.boundary_gradient * p[self.mesh.bface_cell]

    def abs_apply(self, x):
        """Face-factorized |S||x| bound of `_roundoff_residual_floor!`
        (cycles.jl:108-179)."""
        mesh = self.mesh
        ax = np.abs(x)
        face_input = self.sqrt_kappa * mesh.face_area * (ax[mesh.face_minus] + ax[mesh.face_plus])
        face_output = abs(self.K) @ face_input
        bound = mesh.face_area * self.sqrt_kappa * face_output
        out = self.boundary_diagonal * ax
        np.add.at(out, mesh.face_minus, bound)
        np.add.at(out, mesh.face_plus, bound)
        return out


def components(op):
    """Open-face connected components, their volumes and which are ungauged
    (elliptic_solver.jl:39-129; common.jl:53-83).  Returns labels (root cell,
    0-based, -1 for none), anchors (roots of ungauged components, increasing)
    and slots (index into anchors per cell, -1 for none)."""
    mesh = op.mesh
    nc = mesh.ncells
    open_faces = op.face_coefficient != 0
    active = op.volumes > 0
    fm = mesh.face_minus[open_faces]; fp = mesh.face_plus[open_faces]
    G = sp.coo_matrix((np.ones(len(fm)), (fm, fp)), shape=(nc, nc))
    n_comp, lab = sp.csgraph.connected_components(G, directed=False)
    # root = smallest cell index of each component (roots visited in increasing order)
    root_of = np.full(n_comp, nc, dtype=np.int64)
    np.minimum.at(root_of, lab, np.arange(nc))
    labels = np.where(active, root_of[lab], -1)
    # a cell with an open-face conductance anchors its component
    # (elliptic_solver.jl:80-82); the others stay ungauged
    anchored = np.unique(labels[(labels >= 0) & (op.boundary_diagonal != 0)])
    anchors = np.setdiff1d(np.unique(labels[labels >= 0]), anchored)
    slot_of = {int(r): s for s, r in enumerate(anchors)}
    slots = np.array([slot_of.get(int(l), -1) if l >= 0 else -1 for l in labels], dtype=np.int64) \
        if len(anchors) != 1 else np.where(np.isin(labels, anchors), 0, -1)
    comp_volumes = np.array([op.volumes[labels == r].sum() for r in anchors])
    return {"labels": labels, "anchors": anchors, "slots": slots, "volumes": comp_volumes}


def remove_component_volume_means(values, volumes, comp):
    """`_remove_component_volume_means!` (elliptic_solver.jl:132-151)."""
    out = values.copy()
    slots = comp["slots"]
    for s in range(len(comp["anchors"])):
        sel = slots == s
        out[sel] -= np.sum(volumes[sel] * values[sel]) / comp["volumes"][s]
    out[comp["labels"] < 0] = 0.0
    return out


def project_component_rhs(rhs, volumes, comp):
    """`_project_component_rhs!` (elliptic_solver.jl:153-190): returns the
    projected RHS, the removed strong means and their volume-weighted mean."""
    out = rhs.copy()
    slots = comp["slots"]
    means = []
    total, tvol = 0.0, 0.0
    for s in range(len(comp["anchors"])):
        sel = slots == s
        ssum = np.sum(rhs[sel])
        total += ssum
        tvol += comp["volumes"][s]
        mean = ssum / comp["volumes"][s]
        means.append(mean)
        out[sel] -= mean * volumes[sel]
    return out, means, (total / tvol if tvol else 0.0)
