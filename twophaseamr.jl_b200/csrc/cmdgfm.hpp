// Host set-up of the CMDGFM two-block solve: the assembled system's blocks,
// the local Schur complement of the jump block and its incomplete LU, and the
// level schedules the device's triangular solves follow.
//
// The system (two_phase/projection/cmdgfm_projection.jl:1484-1592 assembles
// it in ronaldremmerswaal/TwoPhaseAMR.jl) has n = np + nx rows: np pressure
// increments, one per retained cell of the gauge partition, then nx jumps,
// one per mixed face.  [A B; C J], nonsymmetric.
#pragma once

#include <cstdint>
#include <vector>

namespace tpa {

// CSR with int64 row pointers and sorted int32 columns.
struct CsrRows {
    int64_t n = 0;
    std::vector<int64_t> ptr;
    std::vector<int32_t> col;
    std::vector<double> val;
};

// Rows of a triangular factor in the order of a level schedule: the rows of
// level k are rows[level_ptr[k] .. level_ptr[k+1]), each depending only on
// rows of earlier levels.
struct LevelSchedule {
    std::vector<int32_t> level_ptr;
    std::vector<int32_t> rows;
    int levels() const { return int(level_ptr.size()) - 1; }
};

struct CmdgfmFactor {
    int64_t np = 0, nx = 0;
    CsrRows schur;     // J - C D^-1 B, nx x nx (`_cmdgfm_jump_schur!`)
    CsrRows lower;     // strictly lower L (unit diagonal implied), by rows
    CsrRows upper;     // U without its diagonal, by rows
    std::vector<double> pivot;  // U's diagonal
    CsrRows coupling;  // C: jump rows over pressure columns, nx x np
    LevelSchedule lsched, usched;
    // L^-1 and U^-1 by rows (empty when they outgrew the cap; the device then
    // walks the factors row by row)
    CsrRows linv, uinv;
};

// The inverses of the unit lower `lower` and of `upper` with its pivots, by
// rows.  Column j of an inverse is the solution of L x = e_j (U x = e_j),
// formed by propagating each entry along the factor's columns in solve order;
// an entry smaller than 2^-60 of its column's largest is dropped and not
// propagated, so applying the inverse gives the triangular solve to within
// rounding.  Returns false, with both left empty, when together they would
// exceed `cap` entries.
bool triangular_inverses(const CsrRows& lower, const CsrRows& upper, const std::vector<double>& pivot, int64_t cap,
                         CsrRows& linv, CsrRows& uinv);

// S = J - C D^-1 B (two_phase/projection/cmdgfm_cache.jl:550-610): row f is
// J's entries of row f in column order, then for each C entry (f, c) in
// column order the entries -C[f,c] (B[c,g] / D[c]) of row c, summed into the
// row in that order.  D is the diagonal of the pressure block; a zero or
// missing diagonal is an error.
CsrRows cmdgfm_schur(const CsrRows& m, int64_t np);

// IncompleteLU.jl 0.2 `ilu(A; tau)` (the Crout ILU of Li, Saad and Chow, as
// src/solvers/multigrid/cycles.jl:390-396 calls it): step k forms row k of U,
// A[k, k:] - sum_{i<k} L[k,i] U[i, k:], and column k of L,
// A[k+1:, k] - sum_{i<k} U[i,k] L[k+1:, i], both over i increasing; an entry
// is kept when its magnitude is at least tau (the pivot always) and L's kept
// entries are multiplied by 1 / pivot.  A zero pivot is an error.
void crout_ilu(const CsrRows& a, double tau, CsrRows& lower, CsrRows& upper, std::vector<double>& pivot);

// Level schedules of forward substitution with `lower` and backward
// substitution with `upper`.
LevelSchedule forward_levels(const CsrRows& lower);
LevelSchedule backward_levels(const CsrRows& upper);

// Everything the device solve needs from the system matrix `m` (n x n).
CmdgfmFactor cmdgfm_factor(const CsrRows& m, int64_t np, double tau);

}  // namespace tpa
