// Host-side set-up of the B200 pressure solver: block forest, face schedule,
// inverse face metric, assembled level operators and the tree hierarchy.
//
// These are the integer maps and set-up values that the device solve consumes.
// Every routine states the TwoPhaseAMR.jl function whose result it reproduces
// (paths inside ronaldremmerswaal/TwoPhaseAMR.jl).  Indices are 0-based.
#pragma once

#include <array>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace tpa {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Block key (level, i, j) packed in 64 bits: 6 bits of level, 29 bits per index.
inline uint64_t pack_key(int level, int64_t i, int64_t j) {
    return (uint64_t(level) << 58) | (uint64_t(i) << 29) | uint64_t(j);
}
inline int key_level(uint64_t k) { return int(k >> 58); }
inline int64_t key_i(uint64_t k) { return int64_t((k >> 29) & ((1ull << 29) - 1)); }
inline int64_t key_j(uint64_t k) { return int64_t(k & ((1ull << 29) - 1)); }

// Quadtree forest over a layout of level-0 roots (mesh/topology/mesh.jl:103-110,
// 716-757).  Leaves and internal nodes are kept as key sets.
struct Forest {
    int layout[2] = {1, 1};
    double origin[2] = {0, 0}, extent[2] = {1, 1}, root_extent[2] = {1, 1};
    std::unordered_set<uint64_t> leaves, internal;

    void node_box(uint64_t key, double o[2], double e[2]) const;
    void split(uint64_t key);
    // Leaf covering the level-`level` box (i, j), or 0 when that box is refined
    // further (0 is never a valid leaf key of level > 0 ... a level-0 key (0,0,0)
    // is returned as pack_key(0,0,0) == 0 only via `found`).
    bool leaf_at(int level, int64_t i, int64_t j, uint64_t& out) const;
    void balance(const bool periodic[2]);  // `_balance!` (mesh.jl:673-714)
};

// One rediscretisation level's mesh: sorted leaf blocks of nx x ny cells and the
// axis-major interior / boundary face schedules (mesh.jl:226-246, 759-937).
struct Mesh {
    int base[2] = {16, 16}, bs[2] = {16, 16};
    bool periodic[2] = {true, true};
    double origin[2] = {0, 0}, extent[2] = {1, 1};
    Forest forest;
    std::vector<uint64_t> keys;                   // sorted by (level, j, i)
    std::unordered_map<uint64_t, int32_t> index;  // key -> block
    std::vector<double> bsx, bsy, bvol, box, boy; // spacing, volume, origin per block
    int active = 0;                               // finest active level
    // interior faces (every axis-1 face before every axis-2 face)
    std::vector<int32_t> fm, fp;
    std::vector<int8_t> fax;  // 1 or 2
    std::vector<double> farea;
    // boundary faces
    std::vector<int32_t> bcell;
    std::vector<int8_t> bax, bside;
    std::vector<double> barea;

    int64_t nblocks() const { return int64_t(keys.size()); }
    int64_t cells_per_block() const { return int64_t(bs[0]) * bs[1]; }
    int64_t ncells() const { return nblocks() * cells_per_block(); }
    int64_t nfaces() const { return int64_t(fm.size()); }
    void lattice(int level, int64_t out[2]) const {
        out[0] = int64_t(base[0]) << level;
        out[1] = int64_t(base[1]) << level;
    }
    // `_cell_lattice_bounds` (mesh.jl:450-459)
    void cell_lattice(int64_t cell, const int64_t lat[2], int64_t low[2], int64_t sc[2]) const;
    // `_face_lattice_geometry` (mesh.jl:461-474)
    void face_lattice(int64_t f, const int64_t lat[2], int64_t& normal, int64_t& lo, int64_t& hi) const;
    // its boundary-face form (mesh.jl:476-485)
    void bface_lattice(int64_t b, const int64_t lat[2], int64_t& normal, int64_t& lo, int64_t& hi) const;
    std::vector<double> cell_volumes() const;
};

// Build a mesh from a (possibly unbalanced) leaf set: balance, sort, faces.
// `BlockTreeMesh` constructor (mesh.jl:1059-1121) without the halo schedule.
Mesh build_mesh(const int base[2], const int bs[2], const bool periodic[2], const double origin[2],
                const double extent[2], const std::vector<uint64_t>& leaves);
Mesh mesh_from_forest(Forest forest, const int base[2], const int bs[2], const bool periodic[2]);

// Inverse face metric K: diagonal plus symmetric off-diagonal entries
// (operators/gradient.jl:294-393).
struct Metric {
    std::vector<double> diag;
    std::vector<int32_t> off_row, off_col;  // off-diagonal entries (both triangles)
    std::vector<double> off_val;
    int templates = 0;
    bool diagonal() const { return off_val.empty(); }
};
Metric assemble_metric(const Mesh& mesh);

// CSR matrix with sorted column indices.
struct Csr {
    int64_t n = 0;
    std::vector<int64_t> ptr;
    std::vector<int32_t> col;
    std::vector<double> val;
    double diag(int64_t r) const;
};

// Open-face connected components and the ungauged ones
// (solvers/multigrid/elliptic_solver.jl:1-129; two_phase/projection/common.jl:53-83).
struct Components {
    std::vector<int32_t> slot;    // per cell: ungauged component index or -1
    std::vector<double> volume;   // per ungauged component
    std::vector<int32_t> anchor;  // smallest cell of each ungauged component
};

// Assembled level operator `(A + A')/2` of `J' sqrt(k) K sqrt(k) J`
// (operators/elliptic.jl:157-257, 683-800, 969-980) with its face data.
struct LevelOperator {
    Mesh mesh;
    Metric metric;
    std::vector<double> kappa;  // face coefficient
    std::vector<double> volumes;
    Csr A;
    Components comp;
    bool singular = false;
    // open sides (left, right, bottom, top): pressure Dirichlet 0 on their
    // faces (`_pressure_boundary_sides`, elliptic.jl:76-87)
    bool open[4] = {false, false, false, false};
    std::vector<double> bkappa;  // coefficient per boundary face (used on open faces)
    std::vector<double> bdiag;   // open-face conductance 2 k_b / h |f| per cell (empty: none)
    std::vector<double> bgrad;   // 2 k_b / h per boundary face (0 on closed faces)
    bool any_open() const { return open[0] || open[1] || open[2] || open[3]; }
    bool open_face(int64_t b) const;  // `_pressure_open_face` (elliptic.jl:86-87)
};
// `_boundary_material` (elliptic.jl:91-134): open-face coefficients extended
// from the interior coefficients of the opposite faces (area-weighted).
void extend_boundary_material(LevelOperator& op);
void assemble_operator(LevelOperator& op);

// `_jacobi_weight!` (solvers/multigrid/hierarchy.jl:8-30)
double jacobi_weight(std::vector<double>& inv_diag, const std::vector<double>& row_sums,
                     bool skip_nonpositive, bool allow_zero, bool clamp, double zero_weight);

struct HierarchyOptions {
    int coarse_size = 64, pre_sweeps = 2, post_sweeps = 2, max_levels = 32;
    int smoother = 0;  // 0 damped Jacobi (the reference's), 1 red-black Gauss-Seidel
};

// One level of the tree hierarchy with everything the device V-cycle reads.
struct HostLevel {
    LevelOperator op;
    std::vector<double> inv_diag;  // smoother D^-1 (`_multigrid_level`)
    double weight = 1.0;           // smoother weight (clamped)
    // transfer to the next coarser level: P = (I - wt Dt^-1 A) P_tent
    std::vector<int32_t> owner;        // fine cell -> coarse cell (`_tree_cell_prolongation`)
    std::vector<double> transfer_inv; // Dt^-1 of `_smoothed_transfer_refresh`
    double transfer_weight = 0.0;     // unclamped
    // face-coefficient restriction to the next level (tree_coarsening.jl:347-398)
    std::vector<int64_t> rptr;
    std::vector<int32_t> ridx;
    std::vector<double> rw;
    // the same over the boundary faces (open sides only)
    std::vector<int64_t> brptr;
    std::vector<int32_t> bridx;
    std::vector<double> brw;
};

struct Hierarchy {
    HierarchyOptions opts;
    std::vector<HostLevel> levels;
    // coarsest level: the top-left block of the inverse of the (augmented)
    // matrix `[A v; v' 0]` (geometric_preconditioner.jl:144-169), row-major.
    std::vector<double> coarse_inverse;
    int64_t coarse_n = 0;
};

// `TreeGeometricMultigridPreconditioner(operator; multigrid)` (pruning = :all)
// (geometric_preconditioner.jl:171-442).
Hierarchy build_hierarchy(LevelOperator fine, const HierarchyOptions& opts);
// `_refresh_geometric_multigrid!` (geometric_preconditioner.jl:483-594): new
// fine face coefficients on the fixed topology.
void refresh_hierarchy(Hierarchy& h, const std::vector<double>& kappa);
void finish_level(HostLevel& lev);
void factor_coarse(Hierarchy& h);

}  // namespace tpa
