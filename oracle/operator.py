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

Only the configuration the pressure projection uses is restated: reaction 0,
diffusion 1, no open (Dirichlet) boundary sides and no inactive cells.  Sparse
sums are evaluated by scipy, so assembled values agree with the reference to
rounding, not bitwise.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .metric import assemble_inverse_metric


class PoissonOperator:
    """`PoissonOperator(mesh; face_coefficient)` (elliptic.jl:969-980)."""

    def __init__(self, mesh, face_coefficient=1.0, metric=None):
        self.mesh = mesh
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
        self.refresh(kappa)

    def weighted_metric(self):
        """`M = k K` (diagonal K) or `sqrt(k) K sqrt(k)` (elliptic.jl:185-195)."""
        if self.diagonal_metric:
            return sp.diags(self.face_coefficient * self.K.diagonal())
        s = sp.diags(self.sqrt_kappa)
        return (s @ self.K @ s).tocsc()

    def refresh(self, kappa):
        """`_update_elliptic_face_coefficient!` (elliptic.jl:847-916): new face
        coefficients on the fixed topology."""
        self.face_coefficient = np.asarray(kappa, dtype=np.float64).copy()
        self.sqrt_kappa = np.sqrt(self.face_coefficient)
        A = (self.J.T @ self.weighted_metric() @ self.J).tocsr()
        A = ((A + A.T) / 2).tocsr()
        A.sort_indices()
        self.matrix = A
        self.components = components(self)
        self.singular = len(self.components["anchors"]) > 0
        return self

    def apply(self, x):
        """Factorized action `mul!` (elliptic.jl:1125-1180)."""
        face_input = self.sqrt_kappa * (self.J @ x)
        face_output = self.K @ face_input
        return self.J.T @ (self.sqrt_kappa * face_output)

    def weighted_gradient(self, p):
        """`weighted_gradient!` interior values (elliptic.jl:1272-1297)."""
        jump = self.mesh.face_area * (p[self.mesh.face_plus] - p[self.mesh.face_minus])
        return self.sqrt_kappa * (self.K @ (self.sqrt_kappa * jump))

    def abs_apply(self, x):
        """Face-factorized |S||x| bound of `_roundoff_residual_floor!`
        (cycles.jl:108-179)."""
        mesh = self.mesh
        ax = np.abs(x)
        face_input = self.sqrt_kappa * mesh.face_area * (ax[mesh.face_minus] + ax[mesh.face_plus])
        face_output = abs(self.K) @ face_input
        bound = mesh.face_area * self.sqrt_kappa * face_output
        out = np.zeros(mesh.ncells)
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
    anchors = np.unique(labels[labels >= 0])  # no open Dirichlet faces: all ungauged
    slot_of = {int(r): s for s, r in enumerate(anchors)}
    slots = np.array([slot_of.get(int(l), -1) if l >= 0 else -1 for l in labels], dtype=np.int64) \
        if len(anchors) > 1 else np.where(labels >= 0, 0, -1)
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
