/*
 * tpagmg.h - C-ABI of the B200 pressure-projection solver for TwoPhaseAMR.jl.
 *
 * The library replaces the reference's one-velocity pressure solve: Krylov CG
 * preconditioned by the tree geometric multigrid over the block quadtree, with
 * the variable-coefficient operator -div(kappa grad p) (kappa = 1/rho_f).  All
 * paths cited below are inside ronaldremmerswaal/TwoPhaseAMR.jl.
 *
 * Conventions: indices are 0-based int32 (the reference's are 1-based Int64);
 * cell index = block * nx * ny + j * nx + i with blocks sorted by
 * (level, j, i) (src/mesh/topology/mesh.jl:28-30, 759-773).  The caller owns
 * every host array; the library copies what it needs during the call and keeps
 * no host pointers.  Every call returns a tpa_status; no C++ exception crosses
 * this boundary.  Calls on one context must be serialised by the caller.
 */
#ifndef TPAGMG_H
#define TPAGMG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t tpa_status;
#define TPA_OK 0
#define TPA_ERR_INVALID_ARG 1 /* bad sizes, values or call order (ArgumentError)  */
#define TPA_ERR_CUDA 2        /* CUDA runtime failure or no usable device          */
#define TPA_ERR_TIMEOUT 3     /* a bounded device wait gave up                     */
#define TPA_ERR_NONFINITE 4   /* non-finite input                                  */
#define TPA_ERR_UNSUPPORTED 5 /* outside the supported configuration              */
#define TPA_ERR_STATE 7       /* call made before the state it needs exists        */

#define TPA_PRECISION_FP64 0  /* V-cycle in FP64                                   */
#define TPA_PRECISION_MIXED 1 /* V-cycle in FP32 inside the FP64 CG                */

#define TPA_COMPATIBILITY_PROJECT 0
#define TPA_COMPATIBILITY_ERROR 1

typedef struct tpa_context tpa_context;

/* MultigridOptions (src/solvers/multigrid/options.jl:14-48), plus the
 * smoother: 0 = the reference's damped Jacobi, 1 = red-black Gauss-Seidel
 * (colour (I + J) mod 2 at each cell's own level; red then black before the
 * coarse correction, black then red after it; not in the reference). */
typedef struct {
    int32_t coarse_size; /* default 64 */
    int32_t pre_sweeps;  /* default 2  */
    int32_t post_sweeps; /* default 2  */
    int32_t max_levels;  /* default 32 */
    int32_t smoother;    /* default 0  */
} tpa_multigrid_options;

/* LinearSolverStats (src/solvers/multigrid/stats.jl:15-30) plus device timing. */
typedef struct {
    int32_t cycles;
    int32_t converged;
    int32_t compatible;
    int32_t restarts;
    double initial_l2;
    double initial_linf;
    double final_l2;
    double final_linf;
    double target_linf;
    double residual_scale;
    double removed_rhs_mean;
    double device_ms;       /* CUDA-event time of the solve on the solver stream   */
    int32_t kernel_launches; /* kernels this call launched                         */
    int32_t precision;
    double removed_rhs_max_component_mean; /* max over components of |removed strong mean| */
} tpa_stats;

/* Create a context for CUDA device `device`.  No CUDA call is made until the
 * first device operation.  Replaces the Julia-side EllipticSolver state. */
tpa_status tpa_create(tpa_context** out, int32_t device);
void tpa_destroy(tpa_context* ctx);
/* Message of the last failed call on ctx (valid until the next call). */
const char* tpa_last_error(const tpa_context* ctx);

/* BlockTreeMesh(; base_mesh, block_size, origin, extent, periodic) from its
 * leaf keys (src/mesh/topology/mesh.jl:1059-1121): the library restores 2:1
 * grading (`_balance!`, mesh.jl:673-714), sorts the blocks and builds the face
 * schedules.  leaf_keys holds (level, i, j) per leaf. */
tpa_status tpa_set_mesh(tpa_context* ctx, const int32_t base_mesh[2], const int32_t block_size[2],
                        const int32_t periodic[2], const double origin[2], const double extent[2], int64_t nleaves,
                        const int32_t* leaf_keys);
/* out = {nblocks, ncells, ninterior_faces, nboundary_faces, finest_level}. */
tpa_status tpa_mesh_sizes(const tpa_context* ctx, int64_t out[5]);
/* Sorted leaf keys (3 per block) and geometry (origin x, origin y, spacing x,
 * spacing y, volume per block); either pointer may be NULL
 * (mesh.blocks, mesh.jl:12-19, 759-773). */
tpa_status tpa_mesh_blocks(const tpa_context* ctx, int32_t* keys, double* geometry);
/* Interior faces in schedule order (mesh.faces, mesh.jl:32-38, 874-927):
 * minus cell, plus cell, axis (1 or 2), area.  Any pointer may be NULL. */
tpa_status tpa_mesh_faces(const tpa_context* ctx, int32_t* minus, int32_t* plus, int8_t* axis, double* area);
/* Boundary faces (mesh.boundary_faces, mesh.jl:40-46). */
tpa_status tpa_mesh_boundary_faces(const tpa_context* ctx, int32_t* cell, int8_t* axis, int8_t* side,
                                   double* area);

/* PoissonOperator(mesh; face_coefficient) (src/operators/elliptic.jl:969-980):
 * one nonnegative coefficient per interior face (kappa = 1/rho_f for the
 * two-phase operator, two_phase/forces.jl:113-140). */
tpa_status tpa_set_operator(tpa_context* ctx, const double* face_coefficient);
/* Open (pressure Dirichlet 0) sides, `velocity_boundary` of PoissonOperator:
 * open_sides = {left, right, bottom, top}, nonzero for a side whose velocity
 * condition is Outflow or ZeroGradientVelocity (`_pressure_boundary_sides`,
 * src/operators/elliptic.jl:76-87); periodic axes have none.
 * boundary_coefficient: one per boundary face (tpa_mesh_boundary_faces order,
 * `boundary_face_coefficient`), or NULL to extend the interior coefficients
 * to the open faces (`_boundary_material`, elliptic.jl:91-134).  Each open face
 * adds the conductance 2 k_b / h |f| to its cell's diagonal and anchors that
 * cell's component (`_elliptic_boundary_data!`, elliptic.jl:136-152): such a
 * component has no nullspace and its RHS is not projected.  May be called
 * before or after tpa_set_operator; an existing operator is assembled again
 * and the hierarchy must be rebuilt.  A coefficient refresh keeps the boundary
 * coefficients (`_replace_face_coefficient`, elliptic.jl:809-824) and runs on
 * the host.  The adjoint's face-coefficient gradient holds the boundary
 * coefficients fixed, as a refresh does.  The merged batch rejects operators
 * with open sides (TPA_ERR_UNSUPPORTED). */
tpa_status tpa_set_open_boundaries(tpa_context* ctx, const int32_t open_sides[4], const double* boundary_coefficient);
/* Number of stored off-diagonal inverse-metric entries (0 when K is diagonal),
 * operators/gradient.jl:369-393. */
tpa_status tpa_metric_offdiagonal_count(const tpa_context* ctx, int64_t* count);

/* TreeGeometricMultigridPreconditioner(operator; multigrid) with pruning=:all
 * (src/solvers/multigrid/geometric_preconditioner.jl:171-442); opts may be NULL
 * for the defaults.  Host set-up only. */
tpa_status tpa_build_hierarchy(tpa_context* ctx, const tpa_multigrid_options* opts);
/* Number of levels and the cell count of each (hierarchy.operators). */
tpa_status tpa_hierarchy_sizes(const tpa_context* ctx, int32_t* nlevels, int64_t* sizes, int32_t capacity);
/* Tentative owners of level `level` (fine cell -> coarse cell of level+1),
 * `_tree_cell_prolongation` (tree_coarsening.jl:228-252). */
tpa_status tpa_level_owners(const tpa_context* ctx, int32_t level, int32_t* owners);
/* Level scalars: smoother weight, transfer weight, number of ungauged components. */
tpa_status tpa_level_info(const tpa_context* ctx, int32_t level, double* smoother_weight, double* transfer_weight,
                          int32_t* components);
/* Red-black smoother data of level `level` (host-side, no device call):
 * colour per cell (0 red, 1 black: (I + J) mod 2 at the cell's own level) and
 * the half-sweep weight.  Either output may be NULL. */
tpa_status tpa_level_red_black(const tpa_context* ctx, int32_t level, uint8_t* colours, double* weight);
/* Restricted face coefficients of level `level` (tree_coarsening.jl:538-555). */
tpa_status tpa_level_face_coefficients(const tpa_context* ctx, int32_t level, double* kappa);
/* The assembled operator of level `level`, the stiffness (A + A')/2 with any
 * open-face conductances on its diagonal (operators/elliptic.jl:175-257), as
 * CSR with sorted columns: *nnz receives the entry count; row_ptr (n + 1),
 * col and val (*nnz each) may be NULL to ask for the count first.  Host
 * set-up data, for parity checks and for callers that assemble a larger
 * system around the pressure operator (the CMDGFM system below). */
tpa_status tpa_level_matrix(const tpa_context* ctx, int32_t level, int64_t* nnz, int64_t* row_ptr, int32_t* col,
                            double* val);

/* `_refresh_geometric_multigrid!` (geometric_preconditioner.jl:483-594): new
 * fine face coefficients on the fixed topology; refreshes every level.  Once
 * the hierarchy is on the device, a refresh that keeps the set of zero
 * coefficients runs on the GPU (operator values, both Jacobi weights and the
 * coarse inverse; CSR levels and a coarsest matrix of at most 2048 unknowns);
 * otherwise, or with TPAGMG_HOST_REFRESH set, the host rebuilds the levels and
 * uploads them.  Host-side level queries recompute the host copy on demand. */
tpa_status tpa_refresh(tpa_context* ctx, const double* face_coefficient);
/* tpa_refresh from a device array (e.g. the output of
 * tpa_face_coefficients_device): on the GPU when the set of zero coefficients
 * is unchanged (checked on the device), otherwise the host rebuilds. */
tpa_status tpa_refresh_device(tpa_context* ctx, const double* face_coefficient);
/* How the last tpa_refresh ran: path 1 = on the host, 2 = on the device,
 * 0 = none yet; ms = its host wall time.  Replaces nothing in the reference
 * (measurement support). */
tpa_status tpa_last_refresh(const tpa_context* ctx, int32_t* path, double* ms);

/* solve!(solution, solver, rhs; rtol, atol, max_cycles, compatibility)
 * (src/solvers/multigrid/elliptic_solver.jl:628-675).  rhs is the strong-form
 * right-hand side, x the initial guess on entry and the solution on return,
 * both host arrays in cell order.  precision 0: FP64 V-cycle and Krylov
 * vectors; 1: FP32 V-cycle, FP64 Krylov vectors; 2: FP64 iterative
 * refinement around CG runs whose r, p, Ap and z are stored in FP32 (the
 * iterate, the true residual that starts each run and every inner product
 * stay FP64; a run stops at 1e-5 of the true residual it started from, or at
 * the target).  2 has no counterpart in the reference and needs the default
 * cycle; stats->cycles sums the CG iterations of all runs. */
tpa_status tpa_solve(tpa_context* ctx, const double* rhs, double* x, double rtol, double atol, int32_t max_cycles,
                     int32_t compatibility, int32_t precision, tpa_stats* stats);
/* Same with device pointers (cell order, on the context's device). */
tpa_status tpa_solve_device(tpa_context* ctx, const double* rhs, double* x, double rtol, double atol,
                            int32_t max_cycles, int32_t compatibility, int32_t precision, tpa_stats* stats);

/* Batched uneven solves: solve!(x[k], solver_k, rhs[k]) for `count`
 * independent problems, each with its own context (its own mesh, hierarchy
 * and CUDA stream; contexts must be distinct).  The reference runs such
 * solves one after another (one EllipticSolver per problem, elliptic_solver.jl:
 * 628-675); here up to `workers` host threads (<= 0: 32) keep that many
 * problems in flight on the GPU at once, each problem's CG loop a captured
 * graph on its own stream.  rhs[k] and x[k] are host arrays in the cell order
 * of problem k; stats and statuses (either may be NULL) receive one entry per
 * problem.  All contexts must use one device.  device_ms (may be NULL)
 * receives the device time from a start event, which every problem's stream
 * waits on, to the completion of the last problem.  Returns TPA_OK when every
 * problem succeeded, else the status of the first failed problem (its
 * message: tpa_last_error(ctxs[k])); the other problems are still solved. */
tpa_status tpa_solve_batched(tpa_context* const* ctxs, int32_t count, const double* const* rhs, double* const* x,
                             double rtol, double atol, int32_t max_cycles, int32_t compatibility, int32_t precision,
                             int32_t workers, tpa_stats* stats, tpa_status* statuses, double* device_ms);
/* Same with device pointers (rhs[k], x[k] on the contexts' device). */
tpa_status tpa_solve_batched_device(tpa_context* const* ctxs, int32_t count, const double* const* rhs,
                                    double* const* x, double rtol, double atol, int32_t max_cycles,
                                    int32_t compatibility, int32_t precision, int32_t workers, tpa_stats* stats,
                                    tpa_status* statuses, double* device_ms);

/* Merged batch: the hierarchies of `count` contexts (each after
 * tpa_build_hierarchy, default cycle, one device) merged into one set of batch
 * levels, so that one kernel launch advances a V-cycle phase of every problem
 * (levels aligned at the coarse end; work lists of <= 256 rows that never
 * straddle two problems; per-problem CG scalars and stopping rules; a problem
 * that stops is frozen while the others continue).  Each problem's solve is
 * `solve!` of its own context (elliptic_solver.jl:628-675), which the
 * reference runs one problem at a time.  The batch copies what it needs: the
 * contexts may be changed or destroyed afterwards (a new batch sees the
 * change).  On failure *out still receives a handle holding the message. */
typedef struct tpa_batch tpa_batch;
tpa_status tpa_batch_create(tpa_batch** out, tpa_context* const* ctxs, int32_t count);
void tpa_batch_destroy(tpa_batch* batch);
const char* tpa_batch_last_error(const tpa_batch* batch);
/* out = {problems, fine cells (all problems), batch levels, levels of the per-problem one-CTA tail} */
tpa_status tpa_batch_sizes(const tpa_batch* batch, int64_t out[4]);
/* offsets[k] = first fine cell of problem k in the concatenated arrays (count + 1 entries). */
tpa_status tpa_batch_offsets(const tpa_batch* batch, int64_t* offsets);
tpa_status tpa_batch_set_stream(tpa_batch* batch, void* stream);
/* solve! of every problem: rhs and x are the problems' cell arrays concatenated
 * in problem order (tpa_batch_offsets), host memory.  stats and statuses
 * (NULL or one entry per problem).  A problem rejected before its solve (a
 * nonzero mean with compatibility :error) gets a nonzero status; the others
 * are still solved and the call returns that status. */
tpa_status tpa_batch_solve(tpa_batch* batch, const double* rhs, double* x, double rtol, double atol,
                           int32_t max_cycles, int32_t compatibility, int32_t precision, tpa_stats* stats,
                           tpa_status* statuses);
/* Same with device arrays on the batch's device. */
tpa_status tpa_batch_solve_device(tpa_batch* batch, const double* rhs, double* x, double rtol, double atol,
                                  int32_t max_cycles, int32_t compatibility, int32_t precision, tpa_stats* stats,
                                  tpa_status* statuses);

/* Device layout of the V-cycle (no reference counterpart: the reference's
 * cycle runs on the host).  Negative fields mean "default".  tail_cells: levels
 * with at most this many cells run in the coarse tail; tail_ctas: CTAs of the
 * tail's thread-block cluster (1-8); structured: 0 CSR kernels everywhere, 1
 * stencil kernels on constant-coefficient levels without coarse-fine rows,
 * 2 stencil kernels wherever the transfer has a block map; vectorized: 4-cell
 * kernels on constant-coefficient 16x16 levels; pdl: programmatic dependent
 * launch between cycle kernels; fuse_restrict: on CSR levels (every one for 1,
 * those of at most fuse_restrict cells above 1), the residual is
 * recomputed inside the restriction (one launch instead of two); persistent:
 * when every multi-CTA level is a CSR level, the whole V-cycle runs as one
 * cooperative launch with grid barriers (bounded waits; a barrier that gives up
 * makes the solve return TPA_ERR_TIMEOUT); tiles: 1 (the default) runs each
 * CSR level of the multi-CTA part as two launches on haloed block tiles (both
 * pre-sweeps, the residual and the restriction in one, the prolongation and
 * both post-sweeps in the other; the halo is recomputed in each tile), 2 also
 * the constant-coefficient 16x16 levels (on 22 x 22 stencil tiles), 3 the
 * constant-coefficient levels of at most 2^19 cells only (larger ones keep
 * the vectorized kernels), 4 as 3 with the larger levels of a periodic block
 * lattice (one tree level of 16x16 blocks filling the domain, constant
 * diagonal and volumes) on row-streaming kernels (two launches per level: a
 * warp walks a strip 26 cells wide up the level with the phases one row
 * apart), 5 every periodic lattice level on row-streaming kernels and the
 * other constant-coefficient levels as 3, 0 none.
 * Every layout gives the same V-cycle to rounding. */
typedef struct {
    int32_t tail_cells, tail_ctas, structured, vectorized, pdl, fuse_restrict, persistent, tiles;
    double ms_per_vcycle; /* measured time (tpa_autotune), else 0 */
} tpa_tune_config;
/* Autotuner: times `vcycles` V-cycles (precision 0 FP64, 1 or 2 FP32) of every
 * candidate layout on the uploaded hierarchy (tail size x tail CTAs x stencil
 * policy, then the best without vectorized kernels, without PDL, with the
 * fused restriction, as one cooperative launch and on block tiles), keeps the
 * fastest and returns it in *best; tried (capacity entries, may be NULL)
 * receives every measurement and *ntried their count.  The choice persists
 * across tpa_refresh; a new hierarchy starts from the defaults. */
tpa_status tpa_autotune(tpa_context* ctx, int32_t precision, int32_t vcycles, tpa_tune_config* best,
                        tpa_tune_config* tried, int32_t capacity, int32_t* ntried);
tpa_status tpa_set_tuning(tpa_context* ctx, const tpa_tune_config* config);
/* the layout in effect (defaults resolved; ms_per_vcycle = 0) */
tpa_status tpa_get_tuning(tpa_context* ctx, tpa_tune_config* config);

/* Reverse-mode derivative of tpa_solve (the rrule a Julia caller registers
 * with ChainRulesCore for solve!; the reference differentiates nothing, so
 * the forward map is that of solve!, elliptic_solver.jl:628-675, with
 * compatibility :project).  Given the forward solution p and the cotangent
 * pbar = dJ/dp (host arrays, cell order), it solves the adjoint system (the
 * same symmetric operator, strong right-hand side pbar / V) and returns
 * rhs_bar = dJ/d(strong rhs) = V lam (cells) and kappa_bar = dJ/d(face
 * coefficient) = -lam' (dS/dkappa_f) p (interior faces, tpa_mesh_faces
 * order).  Either output may be NULL.  rtol, atol, max_cycles and precision
 * apply to the adjoint solve; stats describes it.  kappa_bar needs kappa > 0
 * on faces of hanging-vertex patches (TPA_ERR_INVALID_ARG otherwise). */
tpa_status tpa_adjoint(tpa_context* ctx, const double* p, const double* pbar, double* rhs_bar, double* kappa_bar,
                       double rtol, double atol, int32_t max_cycles, int32_t precision, tpa_stats* stats);
/* Same with device pointers (cell and face order, on the context's device). */
tpa_status tpa_adjoint_device(tpa_context* ctx, const double* p, const double* pbar, double* rhs_bar,
                              double* kappa_bar, double rtol, double atol, int32_t max_cycles, int32_t precision,
                              tpa_stats* stats);
/* grad_f = -lam' (dS/dkappa_f) p for given cell vectors p and lam (host
 * arrays): the face kernel of tpa_adjoint on its own.  S is the operator of
 * src/operators/elliptic.jl:157-257 (J' sqrt(k) K sqrt(k) J). */
tpa_status tpa_face_coefficient_gradient(tpa_context* ctx, const double* p, const double* lam, double* grad);

/* y = S x, the integrated pressure operator on the finest level
 * (FactorizedEllipticOperator mul!, elliptic.jl:1125-1180).  Host arrays. */
tpa_status tpa_apply(tpa_context* ctx, const double* x, double* y);
/* z = one V-cycle applied to the integrated residual r (ldiv!, cycles.jl:262-283). */
tpa_status tpa_vcycle(tpa_context* ctx, const double* r, double* z, int32_t precision);
/* Wait for the context's stream. */
tpa_status tpa_synchronize(tpa_context* ctx);
/* `_integrated_residual_norms(r, volumes)` (src/solvers/multigrid/cycles.jl:
 * 210-221, the norms `residual_norms(solver)` reports, elliptic_solver.jl:
 * 677-679) of an integrated residual r on the finest level (device pointer,
 * cell order): out[0] = sqrt(sum_V V (r/V)^2 / sum_V V), out[1] = max |r_i|/V_i
 * over cells of positive volume.  Uses the context's device scratch; out is a
 * host array. */
tpa_status tpa_residual_norms(tpa_context* ctx, const double* r, double out[2]);
/* The same two norms for callers that cannot allocate device memory (memory
 * owned by a pool or arena that must not be bypassed, hosts that forbid
 * runtime allocation).  This entry point has no counterpart in the reference,
 * which has no device code.  r and volumes are device pointers of n cells on
 * the current device; out is a host array.  It calls no cudaMalloc or
 * cudaFree: its scratch is one static device array of about 14 KiB, held by
 * every GPU that loads this library until the process exits.  n must lie in
 * [1, 2^31 - 1]; other sizes are rejected with TPA_ERR_INVALID_ARG before any
 * CUDA call.  The first call on a device looks up the scratch's device address
 * (make that first call before any stream capture); the address is cached for
 * the process and does not survive cudaDeviceReset.  Every call clears the
 * scratch's counter, launches on the legacy default stream and waits for it
 * (a synchronous copy of the two norms).  Every call shares the scratch: calls
 * that overlap on the GPU (from several threads or streams) race and must be
 * serialised by the caller.  ctx is used only for the error message and may
 * be NULL. */
tpa_status tpa_residual_norms_noalloc(tpa_context* ctx, const double* r, const double* volumes, int64_t n,
                                      double out[2]);
/* Device layout of the uploaded hierarchy: out = {levels on the block-
 * structured stencil path, exception (CSR) rows on those levels, first level
 * of the single-CTA coarse tail, 1 if the fused default cycle is used}.
 * Uploads the hierarchy if needed. */
tpa_status tpa_device_info(tpa_context* ctx, int64_t out[4]);
/* Number of levels whose V-cycle phases run on haloed block tiles under the
 * layout in effect (tpa_tune_config.tiles; a level keeps the unfused kernels
 * when its tiles do not fit).  Uploads the hierarchy if needed.  Measurement
 * support; no reference counterpart. */
tpa_status tpa_tiled_levels(tpa_context* ctx, int32_t* count);
/* Of those, the levels on the row-streaming kernels (tpa_tune_config.tiles 4
 * or 5).  Uploads the hierarchy if needed.  Measurement support; no
 * reference counterpart. */
tpa_status tpa_streamed_levels(tpa_context* ctx, int32_t* count);
/* Run subsequent device work on the caller's CUDA stream (a cudaStream_t
 * passed as void*; NULL restores the context's own stream).  Replaces nothing
 * in the reference (it has no device); it lets a caller order the solve with
 * its own device work and time it with events on that stream. */
tpa_status tpa_set_stream(tpa_context* ctx, void* stream);
/* Average device time in ms of `iters` back-to-back launches of one kernel on
 * level `level`: which = 0 smoothing sweep, 1 restriction, 4 first two
 * sweeps, 5 residual (default cycle), 6 / 7 the down / up kernel of a level on
 * CSR tiles, 8 / 9 those of a row-streamed level (tiles 4, 5); on the plain
 * cycle 1 is residual + restriction;
 * 2 prolongation, 3 CG operator product (finest level, FP64).  Measurement
 * support for the roofline; it overwrites the level's work vectors. */
tpa_status tpa_time_kernel(tpa_context* ctx, int32_t which, int32_t level, int32_t precision, int32_t iters,
                           double* ms);

/* ---- the projection step around the solve (device arrays unless noted) ----
 * Face arrays follow the mesh's face order (tpa_mesh_faces), boundary arrays
 * its boundary-face order (tpa_mesh_boundary_faces), cell arrays cell order.
 * All run on the context's stream and return after it has finished. */

/* `_refresh_conditional_fraction!` without embedded geometry
 * (src/interface/interface_field.jl:248-291): the physical fraction clamped to
 * [0, 1] (physical may be NULL) and the conditional fraction with the floor
 * (<= floor -> 0, >= 1 - floor -> 1; the reference's default floor is
 * sqrt(eps)).  TPA_ERR_INVALID_ARG if a value is not finite or lies more than
 * 128 eps outside [0, 1]. */
tpa_status tpa_conditional_fraction_device(tpa_context* ctx, const double* fraction, double fraction_floor,
                                           double* physical, double* conditional);
/* Face coefficients 1/rho_f of `PoissonOperator(field; density)`
 * (src/two_phase/forces.jl:23-36, 69-84, 113-140): rho_f = rho_l c + rho_g (1 - c),
 * c the spacing-weighted mean of the two conditional fractions. */
tpa_status tpa_face_coefficients_device(tpa_context* ctx, const double* conditional, double rho_liquid,
                                        double rho_gas, double* face_coefficient);
/* `surface_tension!` with a constant curvature (forces.jl:179-209, 312-378):
 * jumps sigma * curvature * [c+ > 1/2] - [c- > 1/2] (formulation 0, CGFM) or
 * c+ - c- (1, CSF) times |f|, then sqrt(k) K sqrt(k) of them; boundary
 * values 0 (accel_boundary may be NULL).  Uses the current face coefficients. */
tpa_status tpa_surface_tension_device(tpa_context* ctx, const double* conditional, double sigma, double curvature,
                                      int32_t formulation, double* accel_interior, double* accel_boundary);
/* `weighted_gradient!` (src/operators/elliptic.jl:1255-1297):
 * sqrt(k) K sqrt(k) |f| (p+ - p-) on interior faces; boundary faces carry the
 * zero gradient of a wall (grad_boundary may be NULL). */
tpa_status tpa_weighted_gradient_device(tpa_context* ctx, const double* pressure, double* grad_interior,
                                        double* grad_boundary);
/* `divergence!` (src/operators/advection/cell_advection.jl:205-220). */
tpa_status tpa_divergence_device(tpa_context* ctx, const double* u_interior, const double* u_boundary,
                                 double* divergence);

/* Options of `project!` (src/navier_stokes/projection.jl:183-260). */
typedef struct {
    double dt;                          /* > 0 */
    double tolerance;                   /* in (0, 1); the reference's default is sqrt(eps) */
    double reference_dt;                /* >= dt and finite, or 0 for dt (`_reference_dt`) */
    const double* inherited_divergence; /* NULL, or the `_inherited_divergence` cell array */
    int32_t max_cycles;                 /* default 100 */
    int32_t compatibility;              /* 0 :project, 1 :error */
    int32_t precision;                  /* 0 FP64, 1 mixed, 2 mixed refinement (tpa_solve) */
    int32_t prepared;                   /* 0: `project!` (walls made impermeable first),
                                           1: `_project_prepared!` (boundary velocity as given) */
} tpa_projection_options;

/* `project!` / `_project_prepared!` (projection.jl:221-260): divergence of u,
 * the RHS -div/dt (+ inherited term), the increment solve with rtol 0 and
 * atol tolerance/dt^2, u -= dt G_k phi, p += phi (split domains re-gauged per
 * component).  stats: the solve's, with residual_scale 1/dt^2 and compatible =
 * dt^2 |removed mean| <= tolerance (`_projection_compatibility!`).
 * tpa_project takes host arrays (copied in and out); tpa_project_device takes
 * device arrays (and a device inherited_divergence). */
tpa_status tpa_project(tpa_context* ctx, double* u_interior, double* u_boundary, double* pressure,
                       const tpa_projection_options* options, tpa_stats* stats);
tpa_status tpa_project_device(tpa_context* ctx, double* u_interior, double* u_boundary, double* pressure,
                              const tpa_projection_options* options, tpa_stats* stats);

/* The assembled CMDGFM two-velocity projection system
 * (`_assemble_cmdgfm_system!`, src/two_phase/projection/cmdgfm_projection.jl:
 * 1484-1592): n = np + nx unknowns, the pressure increments of the retained
 * cells of the gauge partition (two_phase/projection/common.jl:89-112), then
 * one jump per mixed face; [A B; C J], nonsymmetric.  Host arrays, 0-based;
 * the pressure unknowns index the context's mesh cells, whose operator (set by
 * tpa_set_operator and tpa_build_hierarchy) is the pressure block's. */
typedef struct {
    int64_t np, nx;
    const int64_t* row_ptr;          /* n + 1 */
    const int32_t* col;              /* row_ptr[n] entries, sorted within a row */
    const double* val;
    const double* rhs;               /* n */
    const int32_t* pressure_cell;    /* np: the cell of each pressure unknown */
    const int32_t* pressure_anchor;  /* np: the anchor cell of its component */
    const double* defect_weight;     /* n: a row's defect is weight |residual| (dt^2 / V for
                                        pressure rows, dt^2 / h for jump rows: `_cmdgfm_residual_defects`) */
    int64_t na;                      /* omitted gauge (anchor) rows, may be 0 */
    const int64_t* extra_row_ptr;    /* na + 1, over the same n unknowns */
    const int32_t* extra_col;
    const double* extra_val;
    const double* extra_rhs;         /* na */
    const double* extra_weight;      /* na (`_cmdgfm_anchor_residual_defect`) */
    const double* row_scale;         /* n: D_r of `_cmdgfm_krylov_scaling!` */
    const double* col_scale;         /* n: D_c */
    double drop_tolerance;           /* incomplete-LU drop tolerance (reference default 1e-3) */
    double tolerance;                /* defect tolerance (reference default sqrt(eps)) */
    int32_t max_iterations;          /* BiCGSTAB iteration budget (reference default 500) */
    int32_t precision;               /* V-cycle: 0 FP64, 1 FP32 */
    const double* initial_pressure;  /* np or NULL: the previous increment in the reduced
                                        unknowns, x[cell] - x[anchor] (`_cmdgfm_initial_solution!`) */
    int32_t warm_start;              /* 1: try zero pressure and then initial_pressure, each with
                                        its jumps from the jump factor, before the Krylov loop
                                        (the reference's default); 0: start from zero */
} tpa_cmdgfm_system;

typedef struct {
    int32_t converged;      /* every defect at or below the tolerance */
    int32_t iterations;     /* BiCGSTAB iterations of all runs */
    int32_t attempts;       /* BiCGSTAB runs */
    int32_t kernel_launches;
    double initial_residual, final_residual;  /* ||rhs||, ||rhs - M x|| */
    double pressure_defect, jump_defect, anchor_defect;
    double setup_ms;        /* host: blocks, Schur complement, incomplete LU, schedules */
    double device_ms;       /* CUDA-event time of the device solve, copies included */
    int64_t factor_entries; /* entries of L and U */
    int32_t lower_levels, upper_levels;  /* depth of the triangular solves */
    int64_t inverse_entries; /* entries of L^-1 and U^-1 when the jump block is applied through
                                them (two parallel products), 0 when the factors are walked row by row */
    int32_t initial_guess_used;  /* the warm start replaced x = 0 */
} tpa_cmdgfm_stats;

/* The linear solve of the CMDGFM projection (`_project_cmdgfm_assembled!`,
 * cmdgfm_projection.jl:2201-2291, without its warm start): residual
 * replacement around BiCGSTAB (Krylov.jl 0.10 `bicgstab!`) on the scaled
 * system D_r M D_c, preconditioned by the block-lower preconditioner of
 * cmdgfm_projection.jl:374-441 -- one V-cycle of the context's pressure
 * hierarchy on the reduced pressure block, then the incomplete LU
 * (IncompleteLU.jl 0.2 `ilu(S; tau)`) of S = J - C D^-1 B
 * (cmdgfm_cache.jl:550-610) on the jump block.  solution: n host doubles.
 * The jump block is limited to 25,600 unknowns (its triangular solves keep
 * the vector in one CTA's shared memory). */
tpa_status tpa_cmdgfm_solve(tpa_context* ctx, const tpa_cmdgfm_system* system, double* solution,
                            tpa_cmdgfm_stats* stats);

/* The host set-up of tpa_cmdgfm_solve alone (no context, no GPU): the Schur
 * complement S (nx x nx) and its incomplete LU, L strictly lower (unit
 * diagonal implied) and U with its diagonal, all CSR with sorted columns.
 * Pass NULL arrays to receive the entry counts (s_nnz, l_nnz, u_nnz) first.
 * Parity checks. */
tpa_status tpa_cmdgfm_factor(const tpa_cmdgfm_system* system, int64_t* s_nnz, int64_t* s_ptr, int32_t* s_col,
                             double* s_val, int64_t* l_nnz, int64_t* l_ptr, int32_t* l_col, double* l_val,
                             int64_t* u_nnz, int64_t* u_ptr, int32_t* u_col, double* u_val);

#ifdef __cplusplus
}
#endif

#endif /* TPAGMG_H */
