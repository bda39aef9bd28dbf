"""Oracle (test infrastructure only): CPU restatement of the linear solve of
TwoPhaseAMR.jl's CMDGFM two-velocity projection, the nonsymmetric two-block
system [A B; C J] [p; xi] = [f; g] in pressure increments p (one per retained
cell of the gauge partition) and face jumps xi (one per mixed face), solved by
BiCGSTAB with a block-lower preconditioner: one tree-GMG V-cycle on the
reduced pressure block, then an incomplete LU of the local Schur complement
J - C D^-1 B on the jump block.

Reference (ronaldremmerswaal/TwoPhaseAMR.jl):
  src/two_phase/projection/common.jl:89-112              `_projection_gauge_partition!`
  src/two_phase/projection/cmdgfm_cache.jl:550-610       `_cmdgfm_jump_schur!` (J - C D^-1 B)
  src/two_phase/projection/cmdgfm_projection.jl:113-236  Krylov scaling: the scaled
      operator D_r M D_c and preconditioner (N^-1 (v / D_r)) / D_c, `_cmdgfm_krylov_scaling!`
  src/two_phase/projection/cmdgfm_projection.jl:374-441  `ldiv!` of the reduced pressure
      and of the block preconditioner
  src/two_phase/projection/cmdgfm_projection.jl:1831-1917 residual defects, the omitted
      gauge (anchor) rows' defect, the scaled residual norm
  src/two_phase/projection/cmdgfm_projection.jl:1951-1971 `_cmdgfm_apply_increment!`
  src/two_phase/projection/cmdgfm_projection.jl:1973-2040 `_cmdgfm_initial_solution!`
      (the warm start; the previous increment is given in the reduced unknowns)
  src/two_phase/projection/cmdgfm_projection.jl:2201-2300 the residual-replacement loop of
      `_project_cmdgfm_assembled!`
  src/solvers/multigrid/cycles.jl:390-396                `incomplete_lu_preconditioner`

Third-party algorithms, absent from the reference tree and restated from their
published descriptions (Project.toml:28-29 pins the versions):
  * Krylov.jl 0.10 `bicgstab!` (van der Vorst's BiCGSTAB, right preconditioner
    N with ldiv, x0 = 0, shadow residual c = b, stop at ||r|| <= atol + rtol ||b||
    or ||r|| + 1 <= 1, breakdown when alpha is 0 or NaN);
  * IncompleteLU.jl 0.2 `ilu(A; tau)`: the Crout ILU of Li, Saad and Chow (row k
    of U and column k of L from the previous ones), an entry kept when its
    magnitude is at least tau before the division by the pivot, every pivot
    kept, L unit lower.
The bits of those two packages are parity unpinned: the restatement fixes the
summation orders that the CUDA path follows, and the tests compare the two
paths on solutions and iteration counts.

The system is given as plain arrays, as the library's C-ABI takes it: the CSR
matrix of the n = np + nx retained rows, the right-hand side, the cell and
anchor cell of every pressure unknown, a defect weight per row (dt^2 / V for
pressure rows, dt^2 / h for jump rows), the omitted anchor rows as CSR rows
over the same unknowns with their right-hand sides and weights, and the
diagonal row and column scalings of `_cmdgfm_krylov_scaling!`.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

EPS = np.finfo(np.float64).eps


@dataclass
class CMDGFMSystem:
    matrix: sp.csr_matrix          # n x n, rows and columns: np pressures, then nx jumps
    rhs: np.ndarray                # n
    np_: int                       # number of pressure unknowns
    pressure_cell: np.ndarray      # np: the cell of each pressure unknown
    pressure_anchor: np.ndarray    # np: the anchor cell of its component
    defect_weight: np.ndarray      # n: row defect = weight * |residual|
    extra: sp.csr_matrix           # na x n: the omitted anchor rows
    extra_rhs: np.ndarray          # na
    extra_weight: np.ndarray       # na
    row_scale: np.ndarray          # n
    col_scale: np.ndarray          # n
    drop_tolerance: float = 1e-3
    tolerance: float = np.sqrt(EPS)
    max_iterations: int = 500
    warm_start: bool = False
    initial_pressure: np.ndarray = None  # np: the previous increment, reduced (x[cell] - x[anchor])

    @property
    def n(self):
        return self.matrix.shape[0]

    @property
    def nx(self):
        return self.n - self.np_


def gauge_partition(labels):
    """`_projection_gauge_partition!` (common.jl:89-112): labels[c] is the root
    (smallest cell) of c's component, or -1 for an inactive cell.  Returns the
    retained cells in increasing order and the anchor of each."""
    labels = np.asarray(labels)
    keep = (labels >= 0) & (labels != np.arange(len(labels)))
    cells = np.nonzero(keep)[0]
    return cells.astype(np.int64), labels[cells].astype(np.int64)


def schur_complement(matrix, np_):
    """`_cmdgfm_jump_schur!` (cmdgfm_cache.jl:550-610): S = J - C D^-1 B with D
    the diagonal of the pressure block.  Row f of S: J's entries of row f in
    column order, then for each C entry (f, c) in column order the entries of
    row c of D^-1 B in column order, each added in that order."""
    M = sp.csr_matrix(matrix)
    n = M.shape[0]
    nx = n - np_
    indptr, indices, data = M.indptr, M.indices, M.data
    diag = np.zeros(np_)
    for c in range(np_):
        for k in range(indptr[c], indptr[c + 1]):
            if indices[k] == c:
                diag[c] = data[k]
    rows = []
    for f in range(nx):
        row = {}
        r = np_ + f
        order = []
        for k in range(indptr[r], indptr[r + 1]):
            j = indices[k]
            if j >= np_:
                g = j - np_
                if g not in row:
                    order.append(g)
                    row[g] = 0.0
                row[g] += data[k]
        for k in range(indptr[r], indptr[r + 1]):
            c = indices[k]
            if c >= np_:
                continue
            cval = data[k]
            for kk in range(indptr[c], indptr[c + 1]):
                j = indices[kk]
                if j < np_:
                    continue
                g = j - np_
                if g not in row:
                    order.append(g)
                    row[g] = 0.0
                row[g] += -(cval * (data[kk] / diag[c]))
        rows.append({g: row[g] for g in sorted(order)})
    return rows  # list of {column: value}, columns increasing


def ilu_crout(rows, tau):
    """IncompleteLU.jl 0.2 `ilu(A; tau)` restated: the Crout ILU.  `rows` is
    the matrix as a list of {column: value} rows.  Returns (L, U): L strictly
    lower by rows ({column: value}, unit diagonal implied), U upper by rows
    (the pivot included).  Step k: u = A[k, k:] - sum_{i<k} L[k,i] U[i, k:]
    over i increasing, l = A[k+1:, k] - sum_{i<k} U[i,k] L[k+1:, i] over i
    increasing; an entry is kept when |value| >= tau (the pivot always), and
    L's kept entries are divided by the pivot."""
    n = len(rows)
    cols = [dict() for _ in range(n)]  # column view of A
    for r, row in enumerate(rows):
        for c, v in row.items():
            cols[c][r] = v
    U = [dict() for _ in range(n)]       # U by rows
    Ucol = [dict() for _ in range(n)]    # U by columns (rows i < column)
    Lrow = [dict() for _ in range(n)]    # L by rows (strictly lower)
    Lcol = [dict() for _ in range(n)]    # L by columns
    for k in range(n):
        u = {c: v for c, v in rows[k].items() if c >= k}
        for i in sorted(Lrow[k]):
            lki = Lrow[k][i]
            for j, uij in U[i].items():
                if j >= k:
                    u[j] = u.get(j, 0.0) - lki * uij
        lc = {r: v for r, v in cols[k].items() if r > k}
        for i in sorted(Ucol[k]):
            uik = Ucol[k][i]
            for r, lri in Lcol[i].items():
                if r > k:
                    lc[r] = lc.get(r, 0.0) - uik * lri
        d = u.get(k, 0.0)
        if d == 0.0:
            raise ZeroDivisionError(f"zero pivot in row {k}")
        for j in sorted(u):
            if j == k or abs(u[j]) >= tau:
                U[k][j] = u[j]
                if j > k:
                    Ucol[j][k] = u[j]
        for r in sorted(lc):
            if abs(lc[r]) >= tau:
                v = lc[r] * (1.0 / d)
                Lcol[k][r] = v
                Lrow[r][k] = v
    return [dict(sorted(r.items())) for r in Lrow], [dict(sorted(r.items())) for r in U]


def ilu_solve(L, U, b):
    """(L U)^-1 b: forward substitution with the unit lower L, then backward
    substitution with U, each row's sum over its columns in increasing order."""
    n = len(L)
    y = np.array(b, dtype=np.float64, copy=True)
    for k in range(n):
        acc = y[k]
        for i, v in L[k].items():
            acc -= v * y[i]
        y[k] = acc
    x = np.zeros(n)
    for k in range(n - 1, -1, -1):
        acc = y[k]
        d = 0.0
        for j, v in U[k].items():
            if j == k:
                d = v
            else:
                acc -= v * x[j]
        x[k] = acc / d
    return x


class ReducedPressure:
    """`ldiv!` of CMDGFMReducedPressurePreconditioner (cmdgfm_projection.jl:
    374-405): the reduced right-hand side scattered to the full cells, each
    anchor collecting minus its component's values in index order, one V-cycle
    of the full-cell hierarchy, and x[cell] - x[anchor] gathered back."""

    def __init__(self, mg, cells, anchors, ncells):
        self.mg, self.cells, self.anchors, self.ncells = mg, np.asarray(cells), np.asarray(anchors), ncells

    def ldiv(self, r):
        full = np.zeros(self.ncells)
        full[self.cells] = 0.0 + r
        for i, a in enumerate(self.anchors):
            full[a] -= r[i]
        sol = self.mg.ldiv(full)
        return sol[self.cells] - sol[self.anchors]


class BlockPreconditioner:
    """`ldiv!` of CMDGFMBlockPreconditioner (cmdgfm_projection.jl:411-441):
    z_p = P^-1 r_p, then z_xi = (L U)^-1 (r_xi - C z_p)."""

    def __init__(self, pressure, matrix, np_, L, U):
        self.pressure, self.np_, self.L, self.U = pressure, np_, L, U
        M = sp.csr_matrix(matrix)
        self.C = M[np_:, :np_]

    def ldiv(self, r):
        np_ = self.np_
        out = np.zeros(len(r))
        if np_ > 0:
            out[:np_] = self.pressure.ldiv(r[:np_])
        if len(r) > np_:
            jr = np.array(r[np_:], dtype=np.float64, copy=True)
            if np_ > 0:
                jr = jr - self.C @ out[:np_]
            out[np_:] = ilu_solve(self.L, self.U, jr)
        return out


def bicgstab(apply_a, apply_n, b, atol, rtol, itmax):
    """Krylov.jl 0.10 `bicgstab!` with the right preconditioner N (ldiv) and
    M = I, started from x = 0 with shadow residual c = b.  Returns (x,
    iterations, status)."""
    n = len(b)
    x = np.zeros(n)
    r = np.array(b, dtype=np.float64, copy=True)
    c = np.array(b, dtype=np.float64, copy=True)
    p = r.copy()
    v = np.zeros(n)
    rnorm = float(np.sqrt(r @ r))
    if rnorm == 0.0:
        return x, 0, "x = 0 is a zero-residual solution"
    eps_stop = atol + rtol * rnorm
    next_rho = float(c @ r)
    if next_rho == 0.0:
        return x, 0, "breakdown: b'c = 0"
    it = 0
    solved = rnorm <= eps_stop
    tired = it >= itmax
    breakdown = False
    N = apply_n if apply_n is not None else (lambda u: u.copy())
    while not (solved or tired or breakdown):
        it += 1
        rho = next_rho
        y = N(p)
        v = apply_a(y)
        alpha = rho / float(c @ v)
        s = r - alpha * v
        x = x + alpha * y
        z = N(s)
        t = apply_a(z)
        omega = float(t @ s) / float(t @ t)
        x = x + omega * z
        r = s - omega * t
        next_rho = float(c @ r)
        beta = (next_rho / rho) * (alpha / omega)
        p = r + beta * (p - omega * v)
        rnorm = float(np.sqrt(r @ r))
        solved = rnorm <= eps_stop or rnorm + 1.0 <= 1.0
        tired = it >= itmax
        breakdown = alpha == 0.0 or np.isnan(alpha)
    status = "solution good enough" if solved else ("breakdown" if breakdown else "maximum iterations")
    return x, it, status


def initial_solution(system, M, pre):
    """`_cmdgfm_initial_solution!` (cmdgfm_projection.jl:1973-2040): two
    candidates, zero pressure and then the previous increment (when given and
    not all zero), each with its jumps from the jump factor,
    (L U)^-1 (rhs_xi - C p); a candidate replaces the best so far when its
    defect is below 0.95 of the best and its scaled residual norm below the
    best's.  Returns (solution, used)."""
    n, npr = system.n, system.np_
    rhs = system.rhs
    best_defect = max(residual_defects(system, rhs))
    best_l2 = float(np.linalg.norm(system.row_scale * rhs))
    solution = np.zeros(n)
    used = False
    for use_previous in (False, True):
        cand = np.zeros(n)
        if use_previous:
            if system.initial_pressure is None:
                continue
            cand[:npr] = system.initial_pressure
            if not np.any(cand[:npr] != 0):
                continue
        if not np.all(np.isfinite(cand[:npr])):
            continue
        if system.nx > 0:
            if pre is None:
                continue
            jr = np.array(rhs[npr:], dtype=np.float64, copy=True) - pre.C @ cand[:npr]
            cand[npr:] = ilu_solve(pre.L, pre.U, jr)
        if not np.all(np.isfinite(cand)):
            continue
        res = rhs - M @ cand
        defect = max(residual_defects(system, res))
        l2 = float(np.linalg.norm(system.row_scale * res))
        if np.isfinite(defect) and np.isfinite(l2) and defect < 0.95 * best_defect and l2 < best_l2:
            solution = cand
            best_defect, best_l2 = defect, l2
            used = True
    return solution, used


@dataclass
class CMDGFMStats:
    converged: bool = False
    initial_guess_used: bool = False
    iterations: int = 0
    attempts: int = 0
    initial_residual: float = 0.0
    final_residual: float = 0.0
    pressure_defect: float = 0.0
    jump_defect: float = 0.0
    anchor_defect: float = 0.0
    history: list = field(default_factory=list)


def residual_defects(system, residual):
    """`_cmdgfm_residual_defects` (cmdgfm_projection.jl:1831-1846): the largest
    weighted pressure-row and jump-row residuals."""
    w = system.defect_weight * np.abs(residual)
    npr = system.np_
    return (float(np.max(w[:npr])) if npr else 0.0, float(np.max(w[npr:])) if system.nx else 0.0)


def anchor_defect(system, solution):
    """`_cmdgfm_anchor_residual_defect` (cmdgfm_projection.jl:1848-1893): the
    omitted gauge rows evaluated at the current solution."""
    if system.extra.shape[0] == 0:
        return 0.0
    res = system.extra_rhs - system.extra @ solution
    return float(np.max(system.extra_weight * np.abs(res)))


def solve(system: CMDGFMSystem, mg, *, preconditioned=True):
    """The linear solve of `_project_cmdgfm_assembled!` (cmdgfm_projection.jl:
    2201-2291), with its warm start when `system.warm_start`: residual replacement around scaled,
    block-preconditioned BiCGSTAB runs.  `mg` is the full-cell hierarchy of the
    pressure operator (its `ldiv` is one V-cycle).  Returns (solution, stats)."""
    M = sp.csr_matrix(system.matrix)
    n, npr = system.n, system.np_
    rows, cols = system.row_scale, system.col_scale
    tol = float(system.tolerance)
    st = CMDGFMStats()
    solution = np.zeros(n)
    st.initial_residual = float(np.linalg.norm(system.rhs))
    pre = None
    if preconditioned:
        S = schur_complement(M, npr)
        L, U = ilu_crout(S, system.drop_tolerance) if system.nx else ([], [])
        ncells = int(max(np.max(system.pressure_cell, initial=-1), np.max(system.pressure_anchor, initial=-1)) + 1)
        ncells = max(ncells, mg.levels[0].n)
        pre = BlockPreconditioner(ReducedPressure(mg, system.pressure_cell, system.pressure_anchor, ncells),
                                  M, npr, L, U)

    def apply_a(v):
        return rows * (M @ (cols * v))

    apply_n = None if pre is None else (lambda v: pre.ldiv(v / rows) / cols)
    correction = np.array(system.rhs, dtype=np.float64, copy=True)
    if n > 0 and st.initial_residual > 0:
        if system.warm_start:
            solution, st.initial_guess_used = initial_solution(system, M, pre)
            correction = system.rhs - M @ solution
        while st.iterations < system.max_iterations:
            pd, jd = residual_defects(system, correction)
            defect = max(pd, jd, anchor_defect(system, solution))
            if not np.isfinite(defect) or defect <= tol:
                break
            srhs = rows * correction
            rhs_norm = float(np.linalg.norm(srhs))
            if not np.isfinite(rhs_norm) or rhs_norm == 0.0:
                break
            requested = min(tol, tol / max(defect, EPS))
            rhs_scale = 1.0
            if rhs_norm < 1.0 and rhs_norm * requested < EPS:
                srhs = srhs / rhs_norm
                rhs_scale = rhs_norm
            itmax = system.max_iterations - st.iterations
            inc, its, _ = bicgstab(apply_a, apply_n, srhs, 0.0, requested, itmax)
            st.iterations += its
            st.attempts += 1
            st.history.append((defect, its))
            if not np.all(np.isfinite(inc)) and pre is not None and st.iterations < system.max_iterations:
                inc, its, _ = bicgstab(apply_a, None, srhs, 0.0, requested,
                                       system.max_iterations - st.iterations)
                st.iterations += its
                st.attempts += 1
            if not np.all(np.isfinite(inc)) or its == 0:
                break
            updated = solution + cols * (rhs_scale * inc)
            changed = bool(np.any(updated != solution))
            solution = updated
            if not changed:
                break
            correction = system.rhs - M @ solution
    st.final_residual = float(np.linalg.norm(correction))
    st.pressure_defect, st.jump_defect = residual_defects(system, correction)
    st.anchor_defect = anchor_defect(system, solution)
    st.converged = max(st.pressure_defect, st.jump_defect, st.anchor_defect) <= tol
    return solution, st
