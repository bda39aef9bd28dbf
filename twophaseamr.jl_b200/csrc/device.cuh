// Device-resident tree hierarchy and the B200 solve (V-cycle + PCG).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "fused.cuh"
#include "host.hpp"
#include "stencil.cuh"
#include "stencil4.cuh"
#include "stream.cuh"
#include "structure.hpp"
#include "tiles.cuh"
#include "tiles.hpp"

namespace tpa {

constexpr int kMaxComponents = 16;
constexpr int kReduceBlocks = 296;   // 2 CTAs per SM on 148 SMs; fixed => deterministic sums
constexpr int kThreads = 256;

#define TPA_CUDA(call)                                                                    \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            throw ::tpa::Error(2, std::string(#call) + ": " + cudaGetErrorString(e_));    \
    } while (0)

template <typename T>
struct DevArray {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        free();
        n = count;
        if (count) TPA_CUDA(cudaMalloc(&p, count * sizeof(T)));
    }
    void upload(const T* h, size_t count, cudaStream_t s) {
        if (count != n) alloc(count);
        if (count) TPA_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void free() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DevArray() { free(); }
    DevArray() = default;
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    DevArray(DevArray&& o) noexcept : p(o.p), n(o.n) {
        o.p = nullptr;
        o.n = 0;
    }
    DevArray& operator=(DevArray&& o) noexcept {
        if (this != &o) {
            free();
            p = o.p;
            n = o.n;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
};

// Level data in one precision T (double for the FP64 cycle, float for the
// mixed-precision cycle).
template <typename T>
struct DevLevelT {
    DevArray<T> val, dinv, tinv, vol;
    DevArray<T> x, y, b, r, s;   // work vectors
    DevArray<T> bp;              // projected right-hand side (fused cycle)
    T w = 1, tw = 0;             // smoother weight, transfer weight
};

struct DevLevel {
    int n = 0, nc = 0;           // cells here, cells on the next coarser level
    int64_t nnz = 0;
    int ncomp = 0;               // ungauged components (0: nonsingular)
    DevArray<int> rowptr, col, owner, child_ptr, child, slot;
    std::vector<double> comp_volume;
    DevLevelT<double> d;
    DevLevelT<float> f;
    DevArray<unsigned char> colour;  // red-black smoother: 0 red, 1 black per cell
    double rbw = 1.0;                // red-black half-sweep weight
    double vol0 = 0;                 // every cell's volume when const_vol
    bool const_vol = false;
    bool any_void = false;           // some cell has volume <= 0 (masked out of sums and rows)
};

// PCG scalars kept on the device between kernels.
struct CgScalars {
    double gamma, gamma_next, pAp, alpha, beta, pnorm2;
    double strong_max, target, rnorm;
    int flags;    // bit0: user exit (strong residual <= target), bit1: zero curvature, bit2: machine/solved
    int iter;
};

// Device layout choices (negative: the default, or the TPAGMG_* environment
// override).  structured: 0 CSR everywhere, 1 stencil path on constant-
// coefficient levels without exception rows, 2 stencil path wherever the block
// map allows it.
struct TuneConfig {
    int tail_cells = -1, tail_ctas = -1, structured = -1, vectorized = -1, pdl = -1;
    int fuse_restrict = -1;  // CSR levels: residual recomputed inside the restriction (0 off,
                             // 1 every level, above 1 levels of at most that many cells)
    int persistent = -1;     // all-CSR hierarchies: the V-cycle as one cooperative launch
    int tiles = -1;          // CSR levels: two launches per level on haloed block tiles (tiles.cuh)
    int tail_smem = -1;      // 1: the coarse tail staged in shared memory (default: global memory)
};

struct SolveStats {
    int cycles = 0, converged = 0;
    double initial_l2 = 0, initial_linf = 0, final_l2 = 0, final_linf = 0, target_linf = 0;
    double residual_scale = 1, removed_rhs_mean = 0;
    double removed_max_component_mean = 0;  // largest |removed strong mean| over the components
    double ms_total = 0;
    int restarts = 0;
};

// CTAs of `fn` (block threads, smem bytes) resident at once on the current
// device: its occupancy times the SM count (cached per kernel and device).
int resident_ctas(const void* fn, int block, size_t smem);

// Grid of a grid-stride launch whose CTAs fold partial sums: every CTA resident
// in one wave (a second wave of a few CTAs would run its whole grid-stride
// share after the first), at most `cap` partials and at most `want` CTAs.
template <typename K>
int fold_grid(K kernel, int block, int64_t want, int cap, size_t smem = 0) {
    const int64_t res = resident_ctas(reinterpret_cast<const void*>(kernel), block, smem);
    return int(std::max<int64_t>(1, std::min<int64_t>(want, std::min<int64_t>(cap, res))));
}

// red-black smoother set-up (device.cu)
std::vector<unsigned char> red_black_colours(const Mesh& m);
double red_black_weight(const Csr& A, const std::vector<unsigned char>& colours);

class DeviceSolver {
public:
    explicit DeviceSolver(int device);
    ~DeviceSolver();
    void upload(const Hierarchy& h);
    int ncells() const { return levels_.empty() ? 0 : levels_[0].n; }
    int nlevels() const { return int(levels_.size()); }
    cudaStream_t stream() const { return stream_; }
    // Run on a caller-owned stream (nullptr: the solver's own stream).
    void set_stream(cudaStream_t s) { stream_ = s ? s : own_stream_; }
    // Average time (ms) of `iters` launches of one kernel family on level `level`:
    // 0 = smoothing sweep, 1 = residual+restriction, 2 = prolongation, 3 = CG operator.
    double time_kernel(int which, int level, int precision, int iters);

    // y = A x on the finest level (FP64), device pointers.
    void apply(const double* x, double* y);
    // z = V-cycle(r), device pointers; precision 0 = FP64, 1 = FP32 cycle.
    void vcycle(const double* r, double* z, int precision);
    // `solve!`: rhs (strong form) and x (initial guess in, solution out) are
    // device pointers in cell order.
    void solve(const double* rhs, double* x, double rtol, double atol, int max_cycles, int compatibility,
               int precision, SolveStats& st);

    // `_integrated_residual_norms` of a finest-level integrated residual
    // (device pointer): out = {L2 of the strong residual, strong L-infinity}.
    void residual_norms(const double* r, double out[2]);

    int kernel_launches() const { return launches_; }
    // changes whenever captured graphs of this solver's kernels go stale (a new
    // upload, a layout, a refresh): callers caching graphs of V-cycles key on it
    unsigned graph_generation() const { return graph_gen_; }
    bool red_black() const { return rb_; }
    void reset_launches() { launches_ = 0; }
    void add_launches(int k) { launches_ += k; }

private:
    template <typename T> DevLevelT<T>& lv(int l);
    template <typename T> void vcycle_t(int l);
    template <typename T> void project_rhs(int l, T* b);
    template <typename T> void remove_means(int l, T* x);
    void strong_max(const double* r, double* out_dev);
    double read_scalar(const double* dev);

    int device_;
    cudaStream_t stream_ = nullptr, own_stream_ = nullptr;
    std::vector<DevLevel> levels_;
    DevArray<double> coarse_inv_, coarse_b_, coarse_x_;
    int coarse_n_ = 0;
    int pre_ = 2, post_ = 2;
    bool rb_ = false;  // red-black Gauss-Seidel smoother in place of damped Jacobi
    // red-black levels up to this many cells fuse each sweep's two half-sweeps
    // into one pass (recomputing the first colour); larger levels use two.
    // Measured slower at every threshold on the droplet (the recomputation
    // costs more than the launch it saves), so 0 unless TPAGMG_RB_PAIR_CELLS.
    int rb_pair_cells_ = 0;
    // fine-level FP64 PCG workspace
    DevArray<double> b_, r_, p_, ap_, z_, tmp_, partial_;
    DevArray<double> bdiag_;   // finest level's open-face conductance per cell (empty: none)
    bool open_sides_ = false;  // the finest operator has an open side
    DevArray<CgScalars> sc_;
    DevArray<double> sums_;   // component sums scratch
    CgScalars* host_sc_ = nullptr;
    double* host_d_ = nullptr;
    int launches_ = 0;
    unsigned graph_gen_ = 0;

    // ---- fused cycle (default options) and the graph-captured CG loop ----
public:
    bool fused() const { return fused_ok_; }
    int tail_first() const { return tail_first_; }

private:
    void build_views();
    template <typename T, typename R> void enqueue_vcycle(const R* r, const double* rsum, double* mean_out);
    template <typename T, typename Epi, typename R>
    void enqueue_vcycle_epi(const R* r, const double* rsum, double* mean_out, const Epi& epi);
    bool rz_foldable() const;
    // CG from the current xw_/b_: returns iterations and flags (Krylov.jl cg! loop)
    void cg_fused(int precision, double target, int itmax, int& niter, int& flags);
    void vcycle_fused(const double* r, double* z, int precision);
    void destroy_graphs();
    cudaGraphExec_t cg_graph(int precision);
    void enqueue_cg_body(int precision, cudaGraphConditionalHandle handle, int set_cond);
    double time_fused(int which, int level, int precision, int iters);

public:
    // Layout (autotune.cu): apply a configuration to the uploaded hierarchy
    // (rebuilds the level views and the stencil copies, not the CSR data).
    void reconfigure(const Hierarchy& h, const TuneConfig& c);
    const TuneConfig& tuning() const { return tune_; }
    void reset_tuning() { tune_ = TuneConfig(); }
    // the configuration actually in effect (defaults and overrides resolved)
    TuneConfig effective_tuning() const;
    // average device time (ms) of `count` V-cycles of a fixed residual
    double time_vcycles(int precision, int count);

private:
    TuneConfig tune_;
    int structured_mode_ = 1;

    // `solve!` with the set-up and checks fused into two passes (solve_fast.cu)
    void solve_fast(const double* rhs, double* x, double rtol, double atol, int max_cycles, int compatibility,
                    int precision, SolveStats& st);
    DevArray<double> spartial_, spres_;
    double vol_total_ = 0;  // finest-level volume of cells with V > 0

    bool fused_ok_ = false;
    bool pdl_ = true;  // programmatic dependent launch between cycle kernels
    int rr_cells_ = 0;  // CSR levels of at most this many cells: residual + restriction in one launch
    int coop_grid_ = 0;     // > 0: the V-cycle runs as one cooperative launch of this many CTAs
    DevArray<unsigned> bar_;  // grid barrier: arrivals, generation
    DevArray<int> err_;       // set when a grid barrier gave up waiting
    unsigned long long barrier_spins_ = 0;  // poll limit of a grid barrier

public:
    // throws (status 3) if a grid barrier of the cooperative V-cycle gave up
    void check_barrier();

private:
    int tail_first_ = 0;
    int tail_ctas_ = 1;  // CTAs of the coarse-tail cluster
    size_t tail_smem_[2] = {0, 0};  // > 0: dynamic shared bytes of the staged tail (FP64, FP32 cycle)
    std::vector<LevelView<double>> vd_;
    std::vector<LevelView<float>> vf_;
    DevArray<LevelView<double>> vd_dev_;
    DevArray<LevelView<float>> vf_dev_;
    DevArray<double> fpartial_, fpartial2_, lsum_, xw_;
    DevArray<unsigned> counters_;
    DevArray<char> cgs_;  // CgState
    // one captured CG loop per precision: 0 FP64, 1 mixed, 2 the refinement
    // solve's inner runs (FP32 r, directions and Ap)
    cudaGraphExec_t cg_exec_[3] = {nullptr, nullptr, nullptr};
    int graph_body_launches_[3] = {0, 0, 0};
    // FP32 r, pa, pb, Ap of the refinement solve, each ir_stride() floats
    // (16-byte aligned sections); allocated by its first solve
    DevArray<float> ir_;
    size_t ir_stride() const { return (size_t(levels_[0].n) + 3) & ~size_t(3); }
    double ir_eta_ = 1e-5;  // inner-run reduction of the refinement solve

    // block-structured level data (stencil + exception rows)
    struct StructDev {
        bool on = false;
        bool vec = false;  // constant-coefficient 16x16 level: vectorized quad kernels (stencil4.cuh)
        DevArray<int> nbr, ex, ex_ptr, ex_col, map;
        DevArray<double> cx_d, cy_d, exv_d;
        DevArray<float> cx_f, cy_f, exv_f;
        int64_t nex = 0;
        bool const_coef = false, const_diag = false;
        int snbx = 0, snby = 0;  // periodic block lattice for the row-streaming kernels (0: none)
    };
    std::vector<StructDev> sdev_;
    std::vector<SView<double>> sd_;
    std::vector<SView<float>> sf_;
    void upload_structured(const Hierarchy& h);

    // haloed block tiles of CSR levels (tiles.hpp, tiles.cuh)
    struct TileDev {
        bool on = false;   // CSR tiles (k_tile_*)
        bool vec = false;  // constant-coefficient 16x16 level: stencil tiles (v_tile_*)
        bool stream = false;  // periodic lattice level: row-streaming kernels (v_stream_*)
        int srows[2] = {0, 0}, sgrid[2] = {0, 0};  // their strip height and grid (FP64, FP32 kernels)
        int cg_rows = 0, cg_grid = 0;              // the same for the CG direction kernel (finest level)
        int ntiles = 0, n3max = 0, n2max = 0, n1max = 0, emax = 0, nent = 0;
        int nt = 256;  // threads per CTA
        DevArray<int> cell, own, cell_off, ring, lrp, lrp_off, ent_off, pos, co, co_off;
        DevArray<int16_t> lcol, ch;
        DevArray<double> val_d;
        DevArray<float> val_f;
    };
    std::vector<TileDev> tdev_;
    StreamGeom stream_geom(int l, bool fp32) const;  // strips of a row-streamed level (stream.cuh)
    StreamGeom stream_cg_geom() const;                // strips of the streamed CG direction kernel
    std::vector<TileView<double>> td_;
    std::vector<TileView<float>> tf_;
    void upload_tiles(const Hierarchy& h);
    template <typename T> const TileView<T>& tile_view(int l) const;
    void gather_tile_values();  // tile copies of the level CSR values (after an upload or a refresh)

public:
    // Levels on the block-structured path and their exception-row counts.
    int structured_levels() const;
    // Levels whose V-cycle phases run on haloed block tiles.
    int tiled_levels() const;
    // Of those, the levels on the row-streaming kernels.
    int streamed_levels() const;
    int64_t exception_rows() const;

    // ---- coefficient refresh on the device (csrc/refresh.cu) ----
    // Largest augmented coarsest matrix the device refresh factors (larger: host path).
    static constexpr int kRefreshMaxCoarse = 2048;
    // The device path applies when no level keeps stencil coefficients of its
    // own and the coarsest matrix is small enough.
    bool refresh_applicable(const Hierarchy& h) const;
    // New finest-level face coefficients (host array, the uploaded topology):
    // every level operator, D^-1, Dt^-1, both weights and the coarse inverse are
    // recomputed on the GPU.  `h` supplies the topology the first time.
    void refresh_on_device(const Hierarchy& h, const double* kappa_host);
    // The same from a device array: 0 when refreshed, 1 when the set of zero
    // coefficients differs from the current one (nothing changed; the host
    // path must rebuild); throws on a non-finite or negative coefficient.
    int refresh_from_device(const Hierarchy& h, const double* kappa_dev);
    // smoother and transfer weight per level, as uploaded or refreshed
    std::vector<double> level_weights();

private:
    struct RefreshLevel {
        int nf = 0, nnz = 0;
        DevArray<int> tptr, tf, tg, rptr, ridx;
        DevArray<double> tc, rw, kappa, sk;
        // block-structured level: CSR positions of the east / north couplings
        // per cell (-1: none) and of the exception rows' entries
        bool structured = false;
        int nex_entries = 0;
        DevArray<int> sx, sy, sex;
    };
    void prepare_refresh(const Hierarchy& h);
    void refresh_levels();  // from the finest coefficients in rl_[0].kappa
    std::vector<RefreshLevel> rl_;
    bool rl_ready_ = false;
    int coarse_N_ = 0, coarse_ncomp_ = 0;
    bool lu_cluster_ = false;  // coarse LU on a cluster with the rows in shared memory
    double* rstage_ = nullptr; // pinned staging of the finest-level coefficients
    DevArray<double> coarse_M_, coarse_MT_, rwtw_, rpart_;
    DevArray<int> coarse_piv_, rerr_;
    DevArray<unsigned> rcnt_;

public:
    // ---- adjoint (csrc/adjoint.cu) ----
    // Finest-level faces, the inverse face metric K as CSR rows (diagonal
    // first) and sqrt(kappa); uploaded on first use and after every refresh.
    void upload_faces(const Mesh& mesh, const Metric& metric, const std::vector<double>& kappa);
    bool faces_ready() const { return nfaces_ >= 0; }
    void invalidate_faces() {
        nfaces_ = -1;
        nbfaces_ = -1;
    }
    int64_t nfaces() const { return nfaces_; }
    // g_f = -lam' (dS/dkappa_f) p for cell vectors p, lam (device pointers).
    void face_gradient(const double* p, const double* lam, double* g);
    // out = in / V (invert = true) or out = in * V on the finest level.
    void scale_by_volume(const double* in, double* out, bool invert);

private:
    int64_t nfaces_ = -1;
    bool hang_zero_ = false;  // a face of a hanging-vertex patch has kappa = 0
    DevArray<int> f_minus_, f_plus_, k_ptr_, k_col_;
    DevArray<double> f_area_, k_val_, f_sqrtk_;

public:
    // ---- the projection step around the solve (csrc/projection.cu) ----
    // Boundary faces, each cell's incident faces in face order and the face
    // spacings (after upload_faces).
    // bgrad: the open-face gradient factor 2 k_b / h per boundary face (0 on
    // closed faces); open: 1 on a face of an open side
    void upload_projection(const Mesh& mesh, const std::vector<double>& bgrad, const std::vector<unsigned char>& open);
    bool has_open_sides() const { return open_sides_; }
    bool projection_ready() const { return nbfaces_ >= 0 && nfaces_ >= 0; }
    int64_t nboundary_faces() const { return nbfaces_; }
    // `_refresh_conditional_fraction!` (no embedded geometry); physical may be null
    void conditional_fraction(const double* raw, double floor, double* physical, double* conditional);
    // kappa_f = 1 / rho_f of `PoissonOperator(field; density)`
    void face_coefficients(const double* conditional, double rho_l, double rho_g, double* kappa);
    // `surface_tension!` with a constant curvature (csf = 0: CGFM)
    void surface_tension(const double* conditional, double sigma, double curvature, int csf, double* a_int,
                         double* a_bnd);
    // `weighted_gradient!` into g (may be null) and / or u -= dt g
    void weighted_gradient(const double* p, double* g_int, double* g_bnd, double* u_int = nullptr,
                           double* u_bnd = nullptr, double dt = 0.0);
    // `divergence!`; rhs: the projection right-hand side -div / dt + weight * inherited
    void divergence(const double* u_int, const double* u_bnd, double* out, bool rhs = false, double dt = 1.0,
                    const double* inherited = nullptr, double weight = 0.0);
    // `project!` (prepared = false: walls made impermeable first) or `_project_prepared!`
    void project(double* u_int, double* u_bnd, double* p, double dt, double tolerance, int max_cycles,
                 int compatibility, const double* inherited, double reference_dt, int precision, bool prepared,
                 SolveStats& st);

private:
    int64_t nbfaces_ = -1;
    DevArray<int> inc_ptr_, inc_code_, b_cell_, perr_;
    DevArray<double> f_hm_, f_hp_, b_side_, b_area_, proj_b_, proj_phi_, proj_in_, proj_part_, proj_cvol_;
    DevArray<double> b_grad_;          // open-face gradient factor per boundary face
    DevArray<unsigned char> b_open_;   // 1 on faces of open sides
};

}  // namespace tpa
