// Fused V-cycle launches and the PCG loop captured as one CUDA graph.
//
// One conjugate-gradient iteration (Krylov.jl 0.10 `cg!` with M = the V-cycle,
// ldiv = true, as called by `_run_krylov!`, src/solvers/multigrid/
// elliptic_solver.jl:403-464 in ronaldremmerswaal/TwoPhaseAMR.jl) is the body
// of a graph WHILE node; the last kernel of the body evaluates the stopping
// rules on the device (machine stop sqrt(r'z) + 1 <= 1, iteration limit, zero
// curvature, and the strong-residual callback max|r_i|/V_i <= target) and sets
// the loop condition, so a whole Krylov run is one graph launch.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "device.cuh"
#include "persistent.cuh"
#include "stream.cuh"
#include "tail_smem.cuh"

namespace tpa {

// the strip height of a row-streamed level: the one whose rounds of resident
// warps (ctas CTAs per SM) walk the fewest rows, the taller on a tie
// (strips of `cols` interior columns; `frame` rows walked besides the interior)
// (`shallow`: the short strips of 8 and 4 rows too, for the small levels,
// where a strip's walk is the kernel's time)
static int stream_rows(int nbx, int nby, int sms, int ctas, int cols = kStreamCols, int frame = 6,
                       bool shallow = true) {
    const int64_t slots = int64_t(ctas) * kStreamWarps * sms;
    int best = 0;
    int64_t cost = 0;
    for (int rows : {36, 24, 16, 8, 4}) {
        if (!shallow && rows < 16) break;
        const int64_t strips = int64_t((16 * nbx + cols - 1) / cols) * ((16 * nby + rows - 1) / rows);
        const int64_t c = (strips + slots - 1) / slots * (rows + frame);
        if (!best || c < cost) {
            best = rows;
            cost = c;
        }
    }
    return best;
}

template <typename F>
static void with_stream_rows(int rows, F f) {
    if (rows == 4) f(std::integral_constant<int, 4>{});
    else if (rows == 8) f(std::integral_constant<int, 8>{});
    else if (rows == 16) f(std::integral_constant<int, 16>{});
    else if (rows == 24) f(std::integral_constant<int, 24>{});
    else f(std::integral_constant<int, 36>{});
}

// the strip heights of the streamed CG direction kernel (finest level)
template <typename F>
static void with_cg_rows(int rows, F f) {
    if (rows == 16) f(std::integral_constant<int, 16>{});
    else if (rows == 24) f(std::integral_constant<int, 24>{});
    else f(std::integral_constant<int, 36>{});
}

namespace {

struct CgState {
    double gamma, pAp, alpha, beta, pnorm2, strong_max, target, rsum, rnorm;
    int flags;  // 1 user exit, 2 zero curvature, 4 machine stop, 8 zero initial residual
    int iter, itmax;
    int fresh;  // the next r'z starts the run (gamma = r'z, p = z)
};

// flags that end a run in the middle of a loop body: the direction and the
// update of that body do nothing
constexpr int kCgHalt = 2 | 4 | 8;

enum Counter { kRestrictSum = 0, kPostMean = 1, kCgAp = 2, kCgUpdate = 3, kCgZ = 4, kCgRes = 5, kRsum = 6 };

inline int blocks_for(int64_t n) {
    int64_t g = (n + kThreads - 1) / kThreads;
    return int(g < 1 ? 1 : g);
}

constexpr int kMaxGrid = 1184;
// tiles = 3: the largest constant-coefficient level on stencil tiles.  A level
// of 2^19 cells is 2048 tiles, under two resident waves of 256-thread CTAs;
// the next level up streams HBM at a rate the tiles' index arithmetic cannot
// keep.
constexpr int kStencilTileCells = 1 << 19;  // 8 CTAs on each of 148 SMs: bounds the partials every fold reads
#define TPA_GRID_STRIDE(i, n) for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

// Kernel launch on `s`, with programmatic dependent launch when `pdl`: the
// next kernel of the cycle is scheduled while this one drains and waits in
// pdl_entry() for its results, which hides the launch gap between the short,
// dependent kernels of a V-cycle.
struct Launch {
    cudaStream_t s;
    bool pdl;
    int cluster = 1;     // CTAs per thread-block cluster (grid must be a multiple)
    bool coop = false;   // cooperative launch (every CTA resident at once)
    template <typename... KArgs, typename... Args>
    void operator()(void (*kernel)(KArgs...), int grid, int block, size_t smem, Args... args) const {
        cudaLaunchConfig_t cfg;
        std::memset(&cfg, 0, sizeof(cfg));
        cfg.gridDim = dim3(unsigned(grid));
        cfg.blockDim = dim3(unsigned(block));
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute at[3];
        unsigned na = 0;
        if (coop) {
            at[na].id = cudaLaunchAttributeCooperative;
            at[na].val.cooperative = 1;
            ++na;
        }
        if (pdl) {
            at[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            at[na].val.programmaticStreamSerializationAllowed = 1;
            ++na;
        }
        if (cluster > 1) {
            at[na].id = cudaLaunchAttributeClusterDimension;
            at[na].val.clusterDim.x = unsigned(cluster);
            at[na].val.clusterDim.y = 1;
            at[na].val.clusterDim.z = 1;
            ++na;
        }
        cfg.attrs = at;
        cfg.numAttrs = na;
        TPA_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
    }
};

// r = b - A x, folds sum(r) into s->rsum
__global__ void k_cg_residual(LevelView<double> A, const double* __restrict__ b, const double* __restrict__ x,
                              double* __restrict__ r, double* partial, unsigned* counter, CgState* s) {
    pdl_entry();
    double v = 0;
    TPA_GRID_STRIDE(i, A.n) {
        double ri = b[i] - rowdot(A, x, i);
        r[i] = ri;
        v += ri;
    }
    if (publish_partial(v, partial, counter)) {
        double t = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            s->rsum = t;
            *counter = 0;
        }
    }
}

__global__ void k_sum_into(int n, const double* __restrict__ v, double* partial, unsigned* counter, double* out) {
    pdl_entry();
    double acc = 0;
    TPA_GRID_STRIDE(i, n) acc += v[i];
    if (publish_partial(acc, partial, counter)) {
        double t = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            *out = t;
            *counter = 0;
        }
    }
}

__device__ __forceinline__ void alpha_from(double pAp, CgState* s) {
    const double eps = 2.220446049250313e-16;
    s->pAp = pAp;
    if (pAp <= eps * s->pnorm2 && fabs(pAp) <= eps * s->pnorm2) {
        s->flags |= 2;
        s->alpha = 0;
    } else {
        s->alpha = s->gamma / pAp;
    }
}

// End of a loop body (Krylov.jl `cg!`: iter += 1, `tired`, then the callback):
// the iteration count, the strong-residual callback max|r_i|/V_i <= target on
// the updated residual, and the loop condition.  A body that halted (zero
// curvature, machine stop, zero initial residual) ends the run uncounted, as
// `cg!` leaves its loop before counting.  One thread.
__device__ __forceinline__ void cg_after_update(CgState* s, bool halted, cudaGraphConditionalHandle handle,
                                                int set_cond) {
    bool stop = halted;
    if (!halted) {
        s->iter += 1;
        if (s->strong_max <= s->target) s->flags |= 1;
        stop = (s->flags & 1) || s->iter >= s->itmax;
    }
    if (set_cond) cudaGraphSetConditional(handle, stop ? 0u : 1u);
}

// Ap = A p and alpha = gamma / p'Ap with the zero-curvature guard: the CG
// operator product alone, as time_fused times it (the CG loop runs the
// *_cg_dir_ap kernels, which also form p)
__global__ void k_cg_ap(LevelView<double> A, const double* __restrict__ p, double* __restrict__ ap, double* partial,
                        unsigned* counter, CgState* s) {
    pdl_entry();
    double v = 0;
    TPA_GRID_STRIDE(i, A.n) {
        double y = rowdot(A, p, i);
        ap[i] = y;
        v += p[i] * y;
    }
    if (publish_partial(v, partial, counter)) {
        double pAp = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            alpha_from(pAp, s);
            *counter = 0;
        }
    }
}

// Search directions of iteration `iter` in the ping-pong pair (pa, pb): the
// previous one (read by the operator product) and the new one (written by it,
// read by the update).
template <typename P>
__device__ __forceinline__ const P* dir_old(const P* pa, const P* pb, int iter) {
    return (iter & 1) ? pb : pa;
}
template <typename P>
__device__ __forceinline__ P* dir_new(P* pa, P* pb, int iter) {
    return (iter & 1) ? pa : pb;
}

// x += alpha p, r -= alpha Ap (p: this iteration's direction); folds
// max|r_i|/V_i and sum(r).  vol null: every cell's volume is vol0.  P is the
// storage type of r, p and Ap (FP32 in the refinement solve's inner runs);
// x and the arithmetic stay FP64, and the norms are those of the stored r.
template <typename P>
__global__ void k_cg_update(int n, double* __restrict__ x, P* __restrict__ r, P* pa, P* pb, const P* __restrict__ ap,
                            const double* __restrict__ vol, double vol0, double* pmax, double* psum,
                            unsigned* counter, CgState* s, cudaGraphConditionalHandle handle, int set_cond) {
    pdl_entry();
    const P* __restrict__ p = dir_new(pa, pb, s->iter);
    __shared__ bool last;
    const bool skip = s->flags & kCgHalt;
    const double alpha = s->alpha;
    double m = 0, sum = 0;
    bool nan = false;
    TPA_GRID_STRIDE(i, n) {
        double ri = double(r[i]);
        if (!skip) {
            x[i] += alpha * double(p[i]);
            const P rs = P(ri - alpha * double(ap[i]));
            r[i] = rs;
            ri = double(rs);
        }
        double V = vol ? vol[i] : vol0;
        if (V > 0) {
            double q = fabs(ri) / V;
            if (q != q) nan = true;
            m = fmax(m, q);
        }
        sum += ri;
    }
    // block max (NaN propagating) and block sum
    __shared__ double shm[32], shs[32];
    __shared__ int nan_seen;
    if (threadIdx.x == 0) nan_seen = 0;
    __syncthreads();
    if (nan) nan_seen = 1;
    double mm = m, ss = sum;
    for (int o = 16; o; o >>= 1) {
        mm = fmax(mm, __shfl_down_sync(0xffffffffu, mm, o));
        ss += __shfl_down_sync(0xffffffffu, ss, o);
    }
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (!lane) {
        shm[wid] = mm;
        shs[wid] = ss;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double bm = 0, bs = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            bm = fmax(bm, shm[w]);
            bs += shs[w];
        }
        pmax[blockIdx.x] = nan_seen ? NAN : bm;
        psum[blockIdx.x] = bs;
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (last) {
        double mx = fold_partials_max(pmax, gridDim.x);
        double sm = fold_partials(psum, gridDim.x);
        if (threadIdx.x == 0) {
            s->strong_max = mx;
            s->rsum = sm;
            *counter = 0;
            cg_after_update(s, skip, handle, set_cond);
        }
    }
}

// block-structured finest level: Ap = A p and alpha
template <int NXC>
__global__ void s_cg_ap(SView<double> L, const double* __restrict__ p, double* __restrict__ ap, double* partial,
                        unsigned* counter, CgState* s) {
    pdl_entry();
    s_apply_dot<double, NXC>(L, p, ap, partial, counter, [&](double pAp) { alpha_from(pAp, s); });
}

// block-structured finest level: r = b - A x, folds sum(r) into s->rsum
template <int NXC>
__global__ void s_cg_residual(SView<double> L, const double* __restrict__ b, const double* __restrict__ x,
                              double* __restrict__ r, double* partial, unsigned* counter, CgState* s) {
    pdl_entry();
    double part = 0;
    for (int bk = blockIdx.x; bk < L.nblocks; bk += gridDim.x) {
        const int t = threadIdx.x;
        const int i = t % Blk<NXC>::nx(L), j = t / Blk<NXC>::nx(L), c = bk * Blk<NXC>::cpb(L) + t;
        double v = b[c] - s_apply<NXC>(L, bk, i, j, c, [&](int q) { return x[q]; });
        r[c] = v;
        part += v;
    }
    if (publish_partial(part, partial, counter)) {
        double tt = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            s->rsum = tt;
            *counter = 0;
        }
    }
}

// constant-coefficient 16x16 finest level: Ap = A p and alpha (vectorized quads)
__global__ void __launch_bounds__(256) v_cg_ap(SView<double> L, const double* __restrict__ p,
                                               double* __restrict__ ap, double* partial, unsigned* counter,
                                               CgState* s) {
    pdl_entry();
    v_apply_dot(L, p, ap, partial, counter, [&](double pAp) { alpha_from(pAp, s); });
}

// constant-coefficient 16x16 finest level: r = b - A x, folds sum(r) into s->rsum
__global__ void __launch_bounds__(256) v_cg_residual(SView<double> L, const double* __restrict__ b,
                                                     const double* __restrict__ x, double* __restrict__ r,
                                                     double* partial, unsigned* counter, CgState* s) {
    pdl_entry();
    const int groups = (L.nblocks + 3) / 4;
    double part = 0;
    for (int grp = blockIdx.x; grp < groups; grp += gridDim.x) {
        const QPos p = q_pos(grp);
        const bool valid = p.b < L.nblocks;
        const QNb<double> g =
            q_gather<double>(L, p, valid, [&](int c) { return q_ldv(x + c); }, [](double v, int) { return v; });
        if (!valid) continue;
        const Quad<double> ax = q_apply(L, g);
        const Quad<double> bb = q_ldv(b + p.c);
        Quad<double> rr;
        for (int m = 0; m < 4; ++m) {
            rr.v[m] = bb.v[m] - ax.v[m];
            part += rr.v[m];
        }
        q_st(r + p.c, rr);
    }
    if (publish_partial(part, partial, counter)) {
        double tt = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            s->rsum = tt;
            *counter = 0;
        }
    }
}

// CTA size of a level's CSR tiles: every tile resident in one wave with as
// many warps per tile as that allows (a tile's phases are dependent chains,
// so its latency falls with the warps that share them)
template <typename F>
void with_tile_threads(int nt, F f) {
    if (nt == 1024) f(std::integral_constant<int, 1024>());
    else if (nt == 512) f(std::integral_constant<int, 512>());
    else f(std::integral_constant<int, 256>());
}

template <typename T, typename F>
void with_nxc(const SView<T>& S, F f) {
    if (S.nx == 16 && S.ny == 16) f(std::integral_constant<int, 16>{});
    else f(std::integral_constant<int, 0>{});
}

__device__ void cg_after_z(CgState* s, double g);

// gamma_next = r'z for z = x0 - mean (the V-cycle's output, not stored: the
// next operator product forms z and p where it reads them), then beta or the
// start of a run (cg_after_z)
template <typename T, typename R>
__global__ void k_cg_z(int n, const T* __restrict__ xv, const double* mean, const R* __restrict__ r,
                       double* partial, unsigned* counter, CgState* s) {
    pdl_entry();
    const double m = mean ? *mean : 0.0;
    double v = 0;
    // whole quads by 16-byte loads (both vectors are allocation-aligned), so a
    // thread keeps 4 cells' loads in flight; then the last n mod 4 cells
    const int nq = n >> 2;
    TPA_GRID_STRIDE(k, nq) {
        const Quad<T> xq = q_ldv(xv + 4 * k);
        const Quad<R> rq = q_ldv(r + 4 * k);
        for (int c = 0; c < 4; ++c) v += double(rq.v[c]) * (double(xq.v[c]) - m);
    }
    for (int i = 4 * nq + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        v += double(r[i]) * (double(xv[i]) - m);
    if (publish_partial(v, partial, counter)) {
        double g = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            *counter = 0;
            cg_after_z(s, g);
        }
    }
}

// gamma_next = g = r'z from the V-cycle at the start of a loop body.  The
// loop body is Krylov.jl's iteration rotated: V-cycle z = M r and r'z, then
// the direction, Ap and alpha, then the x / r update and the stopping rules.
// So a run of k iterations applies k V-cycles; `cg!`'s last z, which only
// its stopping test follows, is not formed.  The iterates and the iteration
// count are those of `cg!`.  A fresh run takes gamma = r'z (zero: nothing to
// solve, flag 8); a later body applies the machine stop sqrt(r'z) + 1 <= 1
// (flag 4; the iteration that reached it was counted by its update) or forms
// beta.  One thread.
__device__ void cg_after_z(CgState* s, double g) {
    if (s->fresh) {
        s->fresh = 0;
        s->gamma = g;
        s->pnorm2 = g;
        s->rnorm = sqrt(g);
        s->beta = 0;
        if (g == 0) s->flags |= 8;
        return;
    }
    const double rnorm = sqrt(g);
    s->rnorm = rnorm;
    if (rnorm + 1.0 <= 1.0) {
        s->flags |= 4;
        return;
    }
    const double beta = g / s->gamma;
    s->beta = beta;
    s->pnorm2 = g + beta * beta * s->pnorm2;
    s->gamma = g;
}

// r'z folded into the finest post-smoothing of the CG loop's V-cycle:
// r'z = sum r_i (x_i - mean) = sum r_i x_i - mean sum r_i, with sum r_i from
// the x / r update (s->rsum)
struct CgRz {
    static constexpr bool kRz = true;
    const double* r;
    double* partial;
    CgState* s;
    __device__ void operator()(double mean, double rx) const { cg_after_z(s, rx - mean * s->rsum); }
};

// The next search direction p = z + beta p_old, formed where the
// operator product reads it: z_j = x_j - mean from the V-cycle's finest-level
// output (FP32 or FP64) and p_old from the other buffer of the ping-pong pair;
// the first iteration of a run (iter 0) takes p = z.  So neither z nor a
// separate p pass goes through memory, and no launch of its own is needed.
// P: the storage type of the directions.  The value is rounded to P where it
// is formed, so the operator product below is that of the stored direction
// (the x update adds the stored one).
template <typename T, typename P>
struct NextDir {
    const T* __restrict__ x;
    const P* __restrict__ pold;
    double mean, beta;
    bool first;
    __device__ __forceinline__ double operator()(int j) const {
        const double z = double(x[j]) - mean;
        return double(P(first ? z : z + beta * double(pold[j])));
    }
};

template <typename T, typename P>
__device__ __forceinline__ NextDir<T, P> next_dir(const T* xv, const double* mean, const P* pa, const P* pb,
                                                  const CgState* s) {
    const int k = s->iter;
    return NextDir<T, P>{xv, dir_old(pa, pb, k), *mean, s->beta, k == 0};
}

// p = z + beta p_old, Ap and alpha = gamma / p'Ap (CSR finest level)
template <typename T, typename P>
__global__ void k_cg_dir_ap(LevelView<double> A, const T* __restrict__ xv, const double* mean, P* pa, P* pb,
                            P* __restrict__ ap, double* partial, unsigned* counter, CgState* s) {
    pdl_entry();
    if (s->flags & kCgHalt) return;  // the run ended at this body's r'z
    const NextDir<T, P> d = next_dir(xv, mean, pa, pb, s);
    P* __restrict__ pn = dir_new(pa, pb, s->iter);
    double v = 0;
    TPA_GRID_STRIDE(i, A.n) {
        double y = 0;
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) y += A.val[k] * d(A.ci[k]);
        const double pi = d(i);
        pn[i] = P(pi);
        ap[i] = P(y);
        v += pi * y;
    }
    if (publish_partial(v, partial, counter)) {
        double pAp = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            alpha_from(pAp, s);
            *counter = 0;
        }
    }
}

// the same on a block-structured finest level
template <typename T, typename P, int NXC>
__global__ void s_cg_dir_ap(SView<double> L, const T* __restrict__ xv, const double* mean, P* pa, P* pb,
                            P* __restrict__ ap, double* partial, unsigned* counter, CgState* s) {
    pdl_entry();
    if (s->flags & kCgHalt) return;  // the run ended at this body's r'z
    const NextDir<T, P> d = next_dir(xv, mean, pa, pb, s);
    P* __restrict__ pn = dir_new(pa, pb, s->iter);
    s_apply_dot_ld<double, NXC>(L, d, [&](int c, double v) { pn[c] = P(v); }, ap, partial, counter,
                                [&](double pAp) { alpha_from(pAp, s); });
}

// the same on a constant-coefficient 16x16 finest level (vectorized quads)
template <typename T, typename P>
__global__ void __launch_bounds__(256) v_cg_dir_ap(SView<double> L, const T* __restrict__ xv, const double* mean,
                                                   P* pa, P* pb, P* __restrict__ ap, double* partial,
                                                   unsigned* counter, CgState* s) {
    pdl_entry();
    if (s->flags & kCgHalt) return;  // the run ended at this body's r'z
    const int k = s->iter;
    const P* __restrict__ po = dir_old(pa, pb, k);
    P* __restrict__ pn = dir_new(pa, pb, k);
    const double mu = *mean, beta = s->beta;
    const bool first = k == 0;
    auto ld = [&](int c) {
        const Quad<T> xq = q_ldv(xv + c);
        Quad<double> q;
        if (first) {
            for (int m = 0; m < 4; ++m) q.v[m] = double(xq.v[m]) - mu;
        } else {
            const Quad<P> pq = q_ldv(po + c);
            for (int m = 0; m < 4; ++m) q.v[m] = (double(xq.v[m]) - mu) + beta * double(pq.v[m]);
        }
        for (int m = 0; m < 4; ++m) q.v[m] = double(P(q.v[m]));  // the stored direction
        return q;
    };
    v_apply_dot_ld(L, ld, pn, ap, partial, counter, [&](double pAp) { alpha_from(pAp, s); });
}

// The same on a periodic lattice finest level, streamed by rows (stream.cuh):
// a warp walks a strip of kStreamCgCols interior columns (a column pair per
// lane, a one-pair frame each side) and ROWS rows with a frame row each side;
// the direction of a row is formed where the row is loaded, and A p one row
// behind it.
constexpr int kStreamCgCols = 60;
constexpr int kStreamCgCtas = 6;  // resident CTAs per SM the kernel is built for

template <typename T, typename P, int ROWS>
__global__ void __launch_bounds__(kStreamWarps * 32, kStreamCgCtas)
    v_stream_dir_ap(SView<double> L, StreamGeom g, const T* __restrict__ xv, const double* mean, P* pa, P* pb,
                    P* __restrict__ ap, double* partial, unsigned* counter, CgState* s) {
    pdl_entry();
    if (s->flags & kCgHalt) return;  // the run ended at this body's r'z
    constexpr int S = ROWS + 2, D = kStreamDepth;
    __shared__ P2<T> sz[kStreamWarps][D][32];
    __shared__ P2<P> sp[kStreamWarps][D][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int it = s->iter;
    const P* __restrict__ po = dir_old(pa, pb, it);
    P* __restrict__ pn = dir_new(pa, pb, it);
    const double mu = *mean, beta = s->beta;
    const bool first = it == 0;
    const int W = g.nbx * 16, H = g.nby * 16;
    double part = 0;
    for (int strip = blockIdx.x * kStreamWarps + wid; strip < g.nsx * g.nsy; strip += gridDim.x * kStreamWarps) {
        const int x0 = (strip % g.nsx) * kStreamCgCols, y0 = (strip / g.nsx) * ROWS;
        const int gx0 = x0 - 2 + 2 * lane;
        const bool out_col = lane >= 1 && lane < 1 + kStreamCgCols / 2 && gx0 < W;
        const int gx = st_wrap(gx0, W);
        auto cell = [&](int k) { return st_cell(g, gx, st_wrap(y0 - 1 + k, H)); };
        auto stage = [&](int k) {
            const int c = cell(k);
            st_cp_async<sizeof(P2<T>)>(&sz[wid][k % D][lane], xv + c);
            if (!first) st_cp_async<sizeof(P2<P>)>(&sp[wid][k % D][lane], po + c);
        };
#pragma unroll
        for (int k = 0; k < D - 1; ++k) {
            stage(k);
            st_commit();
        }
        P2<double> q[S];
#pragma unroll
        for (int k = 0; k < S; ++k) {
            if (k + D - 1 < S) stage(k + D - 1);
            st_commit();
            st_wait<D - 1>();
            const P2<T> z = sz[wid][k % D][lane];
            double ql = double(z.l) - mu, qr = double(z.r) - mu;
            if (!first) {
                const P2<P> pq = sp[wid][k % D][lane];
                ql = (double(z.l) - mu) + beta * double(pq.l);
                qr = (double(z.r) - mu) + beta * double(pq.r);
            }
            q[k] = P2<double>{double(P(ql)), double(P(qr))};  // the stored direction
            if (k >= 2) {  // rows 1 .. ROWS: the interior
                const int j = k - 1;
                const P2<double> ax = st_apply(L, q[j - 1], q[j], q[j + 1]);
                if (out_col && y0 + j - 1 < H) {
                    const int c = cell(j);
                    *reinterpret_cast<P2<P>*>(pn + c) = P2<P>{P(q[j].l), P(q[j].r)};
                    *reinterpret_cast<P2<P>*>(ap + c) = P2<P>{P(ax.l), P(ax.r)};
                    part += q[j].l * ax.l;
                    part += q[j].r * ax.r;
                }
            }
        }
    }
    if (publish_partial(part, partial, counter)) {
        const double sum = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            alpha_from(sum, s);
            *counter = 0;
        }
    }
}

// Start of an inner run of the refinement solve: the FP64 true residual
// rounded to the FP32 recurrence residual, and the sum of the stored values
// (the V-cycle's right-hand-side projection uses it)
__global__ void k_ir_start(int n, const double* __restrict__ r, float* __restrict__ r32, double* partial,
                           unsigned* counter, CgState* s) {
    pdl_entry();
    double v = 0;
    TPA_GRID_STRIDE(i, n) {
        const float ri = float(r[i]);
        r32[i] = ri;
        v += double(ri);
    }
    if (publish_partial(v, partial, counter)) {
        const double t = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            s->rsum = t;
            *counter = 0;
        }
    }
}

__global__ void k_cg_set(CgState* s, double target, int itmax) {
    pdl_entry();
    s->target = target;
    s->itmax = itmax;
    s->flags = 0;
    s->iter = 0;
    s->fresh = 1;
}

__global__ void k_z_out(int n, const float* __restrict__ xf, const double* __restrict__ xd, const double* mean,
                        double* __restrict__ z) {
    pdl_entry();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double m = mean ? *mean : 0.0;
    z[i] = (xf ? double(xf[i]) : xd[i]) - m;
}

}  // namespace

TuneConfig DeviceSolver::effective_tuning() const {
    TuneConfig c;
    c.pdl = tune_.pdl >= 0 ? tune_.pdl : (std::getenv("TPAGMG_NO_PDL") ? 0 : 1);
    c.tail_cells = kTailCellsDefault;
    if (const char* env = std::getenv("TPAGMG_TAIL_CELLS")) c.tail_cells = std::max(0, std::atoi(env));
    if (tune_.tail_cells >= 0) c.tail_cells = tune_.tail_cells;
    c.tail_ctas = kTailCtasDefault;
    if (const char* env = std::getenv("TPAGMG_TAIL_CTAS")) c.tail_ctas = std::atoi(env);
    if (tune_.tail_ctas >= 0) c.tail_ctas = tune_.tail_ctas;
    c.tail_ctas = std::min(8, std::max(1, c.tail_ctas));
    c.structured = 1;
    if (const char* p = std::getenv("TPAGMG_STRUCTURED"))
        if (std::string(p) == "all") c.structured = 2;
    if (std::getenv("TPAGMG_NO_STRUCTURED")) c.structured = 0;
    if (tune_.structured >= 0) c.structured = std::min(2, tune_.structured);
    c.vectorized = std::getenv("TPAGMG_NO_VEC") ? 0 : 1;
    if (tune_.vectorized >= 0) c.vectorized = tune_.vectorized ? 1 : 0;
    c.fuse_restrict = 0;
    if (const char* e = std::getenv("TPAGMG_FUSE_RESTRICT")) c.fuse_restrict = std::max(1, std::atoi(e));
    if (tune_.fuse_restrict >= 0) c.fuse_restrict = tune_.fuse_restrict;
    c.persistent = std::getenv("TPAGMG_PERSISTENT") ? 1 : 0;
    if (tune_.persistent >= 0) c.persistent = tune_.persistent ? 1 : 0;
    // 1: CSR levels on tiles (the default: measured faster on the droplet),
    // 2: the constant-coefficient 16x16 levels on stencil tiles as well
    // (measured slower than the vectorized kernels on uniform 2048^2, whose
    // finest level makes the tile kernel instruction-bound), 3: stencil tiles
    // on the constant-coefficient levels of at most kStencilTileCells cells
    // only, where the six vectorized launches are latency-bound, 4: as 3, with
    // the larger periodic lattice levels on the row-streaming kernels
    // (stream.cuh), 5: every periodic lattice level on the row-streaming
    // kernels, the other constant-coefficient levels as 3, 0: none
    c.tiles = 1;
    if (const char* e = std::getenv("TPAGMG_TILES")) c.tiles = std::min(5, std::max(0, std::atoi(e)));
    if (tune_.tiles >= 0) c.tiles = std::min(5, tune_.tiles);
    if (rb_) {  // the red-black sweeps exist for the CSR levels and the tail only
        c.structured = 0;
        c.persistent = 0;
        c.tiles = 0;
    }
    return c;
}

void DeviceSolver::check_barrier() {
    if (!err_.p) return;
    int e = 0;
    TPA_CUDA(cudaMemcpyAsync(&e, err_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    TPA_CUDA(cudaStreamSynchronize(stream_));
    if (e) {
        TPA_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int), stream_));
        TPA_CUDA(cudaMemsetAsync(bar_.p, 0, 2 * sizeof(unsigned), stream_));
        throw Error(3, "a grid barrier of the cooperative V-cycle gave up waiting; the solve result is invalid");
    }
}

void DeviceSolver::build_views() {
    const TuneConfig cfg = effective_tuning();
    if (const char* e = std::getenv("TPAGMG_RB_PAIR_CELLS")) rb_pair_cells_ = std::atoi(e);
    pdl_ = cfg.pdl != 0;
    // grid-barrier poll limit of the cooperative cycle (TPAGMG_BARRIER_SPINS
    // lowers it; 0 makes every barrier that has to wait give up)
    barrier_spins_ = kBarrierSpins;
    if (const char* e = std::getenv("TPAGMG_BARRIER_SPINS")) barrier_spins_ = std::strtoull(e, nullptr, 10);
    // reduction of the true residual per inner run of the refinement solve
    ir_eta_ = 1e-5;
    if (const char* e = std::getenv("TPAGMG_IR_ETA")) ir_eta_ = std::min(0.5, std::max(1e-7, std::atof(e)));
    // 1: every CSR level; above 1: levels of at most that many cells
    rr_cells_ = cfg.fuse_restrict == 1 ? INT32_MAX : cfg.fuse_restrict;
    fused_ok_ = (pre_ == 2 && post_ == 2);
    for (auto& L : levels_)
        if (L.ncomp > 1) fused_ok_ = false;
    const int nl = int(levels_.size());
    vd_.assign(size_t(nl), LevelView<double>{});
    vf_.assign(size_t(nl), LevelView<float>{});
    const int tail_cells = cfg.tail_cells;
    tail_ctas_ = cfg.tail_ctas;
    tail_first_ = nl - 1;  // the coarsest level always runs in the tail (dense solve)
    for (int l = nl - 1; l >= 0; --l)
        if (levels_[size_t(l)].n <= tail_cells) tail_first_ = l;
        else break;
    int64_t maxgrid = 1;
    for (int l = 0; l < nl; ++l) {
        DevLevel& L = levels_[size_t(l)];
        L.d.bp.alloc(size_t(L.n));
        L.f.bp.alloc(size_t(L.n));
        maxgrid = std::max<int64_t>(maxgrid, blocks_for(L.n));
        auto fill = [&](auto& v, auto& D) {
            v.n = L.n;
            v.nc = L.nc;
            v.rp = L.rowptr.p;
            v.ci = L.col.p;
            v.val = D.val.p;
            v.dinv = D.dinv.p;
            v.tinv = D.tinv.p;
            v.vol = D.vol.p;
            v.owner = L.owner.p;
            v.cptr = L.child_ptr.p;
            v.child = L.child.p;
            v.w = D.w;
            v.tw = D.tw;
            v.singular = L.ncomp == 1;
            v.cvol_inv = L.ncomp == 1 ? 1.0 / L.comp_volume[0] : 0.0;
            v.b = D.b.p;
            v.bp = D.bp.p;
            v.x = D.x.p;
            v.y = D.y.p;
            v.r = D.r.p;
            v.s = D.s.p;
            v.colour = L.colour.p;
            v.rb = rb_ ? 1 : 0;
            v.rbw = static_cast<decltype(v.w)>(L.rbw);
            v.bdiag = nullptr;
        };
        fill(vd_[size_t(l)], L.d);
        fill(vf_[size_t(l)], L.f);
        if (l == 0) vd_[0].bdiag = bdiag_.p;
    }
    vd_dev_.upload(vd_.data(), vd_.size(), stream_);
    vf_dev_.upload(vf_.data(), vf_.size(), stream_);
    // the coarse tail staged in shared memory when its levels fit (one CTA,
    // Jacobi), on request only (TPAGMG_TAIL_SMEM or tail_smem = 1): measured on
    // the droplet its copy-in costs more than the global-load chains it removes
    // (V-cycle 101.6 against 97.9 us)
    tail_smem_[0] = tail_smem_[1] = 0;
    const bool want_tail_smem = tune_.tail_smem >= 0 ? tune_.tail_smem != 0 : std::getenv("TPAGMG_TAIL_SMEM") != nullptr;
    if (fused_ok_ && !rb_ && tail_ctas_ == 1 && nl <= kTailSmemMaxLevels && want_tail_smem) {
        size_t bd = 0, bf = 0;
        for (int l = tail_first_; l < nl; ++l) {
            const DevLevel& L = levels_[size_t(l)];
            const bool last = l == nl - 1;
            bd += tail_level_bytes<double>(L.n, int(L.nnz), last ? 0 : L.nc, last);
            bf += tail_level_bytes<float>(L.n, int(L.nnz), last ? 0 : L.nc, last);
        }
        int optin = 0;
        TPA_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_));
        // room for the kernel's static shared memory (views, reductions)
        const size_t room = size_t(optin) > 16384 ? size_t(optin) - 16384 : 0;
        if (bd <= room) {
            TPA_CUDA(cudaFuncSetAttribute(k_tail_smem<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(bd)));
            tail_smem_[0] = bd;
        }
        if (bf <= room) {
            TPA_CUDA(cudaFuncSetAttribute(k_tail_smem<float, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(bf)));
            tail_smem_[1] = bf;
        }
    }
    // every folding launch has at most max(maxgrid, kMaxGrid) CTAs
    fpartial_.alloc(size_t(std::max<int64_t>(maxgrid, kMaxGrid)));
    fpartial2_.alloc(size_t(std::max<int64_t>(maxgrid, kMaxGrid)));
    lsum_.alloc(size_t(nl + 2));
    xw_.alloc(size_t(levels_[0].n));
    counters_.alloc(16);
    TPA_CUDA(cudaMemsetAsync(counters_.p, 0, 16 * sizeof(unsigned), stream_));
    TPA_CUDA(cudaMemsetAsync(lsum_.p, 0, size_t(nl + 2) * sizeof(double), stream_));
    cgs_.alloc(sizeof(CgState));
    TPA_CUDA(cudaMemsetAsync(cgs_.p, 0, sizeof(CgState), stream_));
    spartial_.alloc(size_t(4) * size_t(kMaxGrid));
    spres_.alloc(8);
    bar_.alloc(2);
    err_.alloc(1);
    TPA_CUDA(cudaMemsetAsync(bar_.p, 0, 2 * sizeof(unsigned), stream_));
    TPA_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int), stream_));
    TPA_CUDA(cudaStreamSynchronize(stream_));
    destroy_graphs();
}

void DeviceSolver::destroy_graphs() {
    ++graph_gen_;
    for (auto& g : cg_exec_)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

// V-cycle on r (integrated residual, FP64 or FP32 storage R) with level-0
// RHS sum `rsum` (device pointer); result in view 0's x, level-0 mean in
// *mean_out.
template <typename T, typename R>
void DeviceSolver::enqueue_vcycle(const R* r, const double* rsum, double* mean_out) {
    enqueue_vcycle_epi<T>(r, rsum, mean_out, MeanOnly());
}

// The same, with `epi` run by the finest level's last post-smoothing after it
// folds the mean (see MeanOnly).  The caller checks rz_foldable() first when
// the epilogue must run.
template <typename T, typename Epi, typename R>
void DeviceSolver::enqueue_vcycle_epi(const R* r, const double* rsum, double* mean_out, const Epi& epi) {
    const Launch go{stream_, pdl_};
    const int nl = int(levels_.size());
    const int t = tail_first_;
    const std::vector<LevelView<T>>* Vp;
    const LevelView<T>* Vdev;
    if constexpr (std::is_same<T, double>::value) {
        Vp = &vd_;
        Vdev = vd_dev_.p;
    } else {
        Vp = &vf_;
        Vdev = vf_dev_.p;
    }
    const std::vector<LevelView<T>>& V = *Vp;
    if (coop_grid_ > 0) {
        // the whole cycle in one cooperative launch (persistent.cuh)
        if constexpr (std::is_same<R, double>::value) {
            const Launch gc{stream_, false, 1, true};
            gc(k_vcycle_grid<T>, coop_grid_, kTailThreads, 0, Vdev, t, nl, r, rsum, mean_out, coarse_inv_.p,
               coarse_n_, fpartial_.p, bar_.p, lsum_.p, err_.p, barrier_spins_);
            ++launches_;
        } else {
            throw Error(5, "the cooperative V-cycle takes an FP64 right-hand side");
        }
        if (!V[0].singular) TPA_CUDA(cudaMemsetAsync(mean_out, 0, sizeof(double), stream_));
        return;
    }
    const std::vector<SView<T>>* Sp;
    if constexpr (std::is_same<T, double>::value) Sp = &sd_;
    else Sp = &sf_;
    for (int l = 0; l < t; ++l) {
        const LevelView<T>& L = V[size_t(l)];
        if (sdev_[size_t(l)].vec) {
            const SView<T>& S = (*Sp)[size_t(l)];
            const int groups = (S.nblocks + 3) / 4;
            const bool next_sum = (l + 1 < t) && V[size_t(l + 1)].singular;
            if (tdev_.size() > size_t(l) && tdev_[size_t(l)].stream) {
                // both pre-sweeps, the residual and the restriction, streamed by rows
                constexpr bool fp32 = std::is_same<T, float>::value;
                const StreamGeom g = stream_geom(l, fp32);
                const int grid = tdev_[size_t(l)].sgrid[fp32 ? 1 : 0];
                with_stream_rows(g.rows, [&](auto rows) {
                    constexpr int RW = decltype(rows)::value;
                    if (l == 0)
                        go(v_stream_down<T, R, RW>, grid, kStreamWarps * 32, 0, S, g, r, rsum, V[size_t(l + 1)].b,
                           fpartial_.p, counters_.p + kRestrictSum, next_sum ? lsum_.p + l + 1 : nullptr);
                    else
                        go(v_stream_down<T, T, RW>, grid, kStreamWarps * 32, 0, S, g, (const T*)S.b,
                           (const double*)(lsum_.p + l), V[size_t(l + 1)].b, fpartial_.p,
                           counters_.p + kRestrictSum, next_sum ? lsum_.p + l + 1 : nullptr);
                });
                ++launches_;
                continue;
            }
            if (tdev_.size() > size_t(l) && tdev_[size_t(l)].vec) {
                // both pre-sweeps, the residual and the restriction on 22 x 22 tiles
                if (l == 0)
                    go(v_tile_down<T, R>, S.nblocks, kTileThreads, 0, S, r, rsum, V[size_t(l + 1)].b, fpartial_.p,
                       counters_.p + kRestrictSum, next_sum ? lsum_.p + l + 1 : nullptr);
                else
                    go(v_tile_down<T, T>, S.nblocks, kTileThreads, 0, S, (const T*)S.b,
                       (const double*)(lsum_.p + l), V[size_t(l + 1)].b, fpartial_.p, counters_.p + kRestrictSum,
                       next_sum ? lsum_.p + l + 1 : nullptr);
                ++launches_;
                continue;
            }
            if (l == 0) go(v_pre2<T, R>, groups, 256, 0, S, r, rsum);
            else go(v_pre2<T, T>, groups, 256, 0, S, S.b, lsum_.p + l);
            go(v_residual<T>, groups, 256, 0, S);
            go(v_restrict<T>, next_sum ? fold_grid(v_restrict<T>, 256, groups, kMaxGrid) : groups, 256, 0, S,
               V[size_t(l + 1)].b,
               fpartial_.p, counters_.p + kRestrictSum, next_sum ? lsum_.p + l + 1 : nullptr);
            launches_ += 3;
            continue;
        }
        if (sdev_[size_t(l)].on) {
            const SView<T>& S = (*Sp)[size_t(l)];
            const int g = S.nblocks, th = S.cpb;
            const bool next_sum = (l + 1 < t) && V[size_t(l + 1)].singular;
            with_nxc(S, [&](auto nxc) {
                constexpr int N = decltype(nxc)::value;
                if (l == 0) go(s_pre2<T, R, N>, g, th, 0, S, r, rsum);
                else go(s_pre2<T, T, N>, g, th, 0, S, S.b, lsum_.p + l);
                go(s_residual<T, N>, g, th, 0, S);
                go(s_restrict<T, N>, next_sum ? fold_grid(s_restrict<T, N>, th, g, kMaxGrid, th * sizeof(T)) : g,
                   th, th * sizeof(T),
                    S, V[size_t(l + 1)].b, fpartial_.p, counters_.p + kRestrictSum,
                    next_sum ? lsum_.p + l + 1 : nullptr);
            });
            launches_ += 3;
            continue;
        }
        if (tdev_.size() > size_t(l) && tdev_[size_t(l)].on) {
            // both pre-sweeps, the residual and the restriction in one launch
            const TileDev& D = tdev_[size_t(l)];
            const TileView<T>& TV = tile_view<T>(l);
            const bool next_sum = (l + 1 < t) && V[size_t(l + 1)].singular;
            const size_t sm = tile_down_smem<T>(D.n3max, D.n2max, D.n1max, D.emax);
            with_tile_threads(D.nt, [&](auto nt) {
                constexpr int NT = decltype(nt)::value;
                if (l == 0)
                    go(k_tile_down<T, R, NT>, D.ntiles, NT, sm, L, TV, r, rsum, V[size_t(l + 1)].b, fpartial_.p,
                       counters_.p + kRestrictSum, next_sum ? lsum_.p + l + 1 : nullptr);
                else
                    go(k_tile_down<T, T, NT>, D.ntiles, NT, sm, L, TV, (const T*)L.b, (const double*)(lsum_.p + l),
                       V[size_t(l + 1)].b, fpartial_.p, counters_.p + kRestrictSum,
                       next_sum ? lsum_.p + l + 1 : nullptr);
            });
            ++launches_;
            continue;
        }
        if (L.rb) {
            // second sweep: one pass on a small level (the red values recomputed),
            // two half-sweeps on a large one
            const bool pair = L.n <= rb_pair_cells_;
            T* first = pair ? L.y : L.x;
            if (l == 0) go(k_rb_pre<T, R>, blocks_for(L.n), kThreads, 0, L, r, rsum, first);
            else go(k_rb_pre<T, T>, blocks_for(L.n), kThreads, 0, L, L.b, lsum_.p + l, first);
            if (pair) {
                go(k_rb_pair<T>, blocks_for(L.n), kThreads, 0, L, (const T*)L.y, L.x, 0, nullptr, nullptr, nullptr);
                ++launches_;
            } else {
                go(k_rb_half<T>, blocks_for(L.n), kThreads, 0, L, (const T*)L.x, L.y, 0, nullptr, nullptr, nullptr);
                go(k_rb_half<T>, blocks_for(L.n), kThreads, 0, L, (const T*)L.y, L.x, 1, nullptr, nullptr, nullptr);
                launches_ += 2;
            }
        } else if (l == 0) {
            go(k_pre2<T, R>, blocks_for(L.n), kThreads, 0, L, r, rsum);
        } else {
            go(k_pre2<T, T>, blocks_for(L.n), kThreads, 0, L, L.b, lsum_.p + l);
        }
        const bool next_sum = (l + 1 < t) && V[size_t(l + 1)].singular;
        const int64_t quads = blocks_for(4 * int64_t(L.nc));
        const int rgrid = !next_sum ? int(quads)
                          : L.n <= rr_cells_ ? fold_grid(k_resrest<T>, kThreads, quads, kMaxGrid)
                                     : fold_grid(k_restrict<T>, kThreads, quads, kMaxGrid);
        if (L.n <= rr_cells_) {
            go(k_resrest<T>, rgrid, kThreads, 0, L, V[size_t(l + 1)].b, fpartial_.p, counters_.p + kRestrictSum,
               next_sum ? lsum_.p + l + 1 : nullptr);
            launches_ += 2;
            continue;
        }
        go(k_residual<T>, blocks_for(L.n), kThreads, 0, L);
        go(k_restrict<T>, rgrid, kThreads, 0, L, V[size_t(l + 1)].b, fpartial_.p, counters_.p + kRestrictSum,
           next_sum ? lsum_.p + l + 1 : nullptr);
        launches_ += 3;
    }
    const size_t tsm = tail_smem_[std::is_same<T, double>::value ? 0 : 1];
    if (tsm > 0) {
        // the tail's levels staged in shared memory (tail_smem.cuh)
        go(k_tail_smem<T, R>, 1, kTailThreads, tsm, Vdev, t, nl, t == 0 ? r : nullptr, coarse_inv_.p, coarse_n_,
           t == 0 && V[0].singular ? mean_out : nullptr);
        ++launches_;
    } else {
    const Launch gt{stream_, pdl_, tail_ctas_};
    gt(k_tail<T, R>, tail_ctas_, kTailThreads, 0, Vdev, t, nl, t == 0 ? r : nullptr, coarse_inv_.p, coarse_n_,
                                                         t == 0 && V[0].singular ? mean_out : nullptr);
    ++launches_;
    }
    for (int l = t - 1; l >= 0; --l) {
        const LevelView<T>& L = V[size_t(l)];
        if (sdev_[size_t(l)].vec) {
            const SView<T>& S = (*Sp)[size_t(l)];
            const int groups = (S.nblocks + 3) / 4;
            const bool want_mean = (l == 0) && L.singular;
            if (tdev_.size() > size_t(l) && tdev_[size_t(l)].stream) {
                // prolongation and both post-sweeps, streamed by rows
                constexpr bool fp32 = std::is_same<T, float>::value;
                const StreamGeom g = stream_geom(l, fp32);
                const int grid = tdev_[size_t(l)].sgrid[fp32 ? 1 : 0];
                with_stream_rows(g.rows, [&](auto rows) {
                    constexpr int RW = decltype(rows)::value;
                    go(v_stream_up<T, Epi, RW>, grid, kStreamWarps * 32, 0, S, g, (const T*)V[size_t(l + 1)].x,
                       fpartial_.p, counters_.p + kPostMean, want_mean ? mean_out : nullptr, epi);
                });
                ++launches_;
                continue;
            }
            if (tdev_.size() > size_t(l) && tdev_[size_t(l)].vec) {
                // prolongation and both post-sweeps on 22 x 22 tiles
                go(v_tile_up<T, Epi>, S.nblocks, kTileThreads, 0, S, (const T*)V[size_t(l + 1)].x, fpartial_.p,
                   counters_.p + kPostMean, want_mean ? mean_out : nullptr, epi);
                ++launches_;
                continue;
            }
            go(v_prolong<T>, groups, 256, 0, S, V[size_t(l + 1)].x);
            go(v_sweep<T, false>, groups, 256, 0, S, S.x, S.y, nullptr, nullptr, nullptr, MeanOnly());
            if (want_mean)
                go(v_sweep<T, true, Epi>, fold_grid(v_sweep<T, true, Epi>, 256, groups, kMaxGrid), 256, 0, S, S.y,
                   S.x, fpartial_.p, counters_.p + kPostMean, mean_out, epi);
            else
                go(v_sweep<T, false>, groups, 256, 0, S, S.y, S.x, nullptr, nullptr, nullptr, MeanOnly());
            launches_ += 3;
            continue;
        }
        if (sdev_[size_t(l)].on) {
            const SView<T>& S = (*Sp)[size_t(l)];
            const int g = S.nblocks, th = S.cpb;
            const bool want_mean = (l == 0) && L.singular;
            with_nxc(S, [&](auto nxc) {
                constexpr int N = decltype(nxc)::value;
                go(s_prolong<T, N>, g, th, 0, S, V[size_t(l + 1)].x);
                go(s_post1<T, N>, g, th, 0, S);
                go(s_post2<T, N, Epi>, want_mean ? fold_grid(s_post2<T, N, Epi>, th, g, kMaxGrid) : g, th, 0, S,
                   fpartial_.p, counters_.p + kPostMean, want_mean ? mean_out : nullptr, epi);
            });
            launches_ += 3;
            continue;
        }
        if (tdev_.size() > size_t(l) && tdev_[size_t(l)].on) {
            // prolongation and both post-sweeps in one launch
            const TileDev& D = tdev_[size_t(l)];
            const bool want_mean = (l == 0) && L.singular;
            with_tile_threads(D.nt, [&](auto nt) {
                constexpr int NT = decltype(nt)::value;
                go(k_tile_up<T, Epi, NT>, D.ntiles, NT, tile_up_smem<T>(D.n3max, D.n2max, D.n1max, D.emax), L,
                   tile_view<T>(l), (const T*)V[size_t(l + 1)].x, fpartial_.p, counters_.p + kPostMean,
                   want_mean ? mean_out : nullptr, epi);
            });
            ++launches_;
            continue;
        }
        go(k_prolong<T>, blocks_for(L.n), kThreads, 0, L, V[size_t(l + 1)].x);
        if (L.rb) {
            const bool last_mean = (l == 0) && L.singular;
            double* mo = last_mean ? mean_out : nullptr;
            if (L.n <= rb_pair_cells_) {
                go(k_rb_pair<T>, blocks_for(L.n), kThreads, 0, L, (const T*)L.x, L.y, 1, nullptr, nullptr, nullptr);
                go(k_rb_pair<T>, blocks_for(L.n), kThreads, 0, L, (const T*)L.y, L.x, 1, fpartial_.p,
                   counters_.p + kPostMean, mo);
                launches_ += 3;
            } else {
                go(k_rb_half<T>, blocks_for(L.n), kThreads, 0, L, (const T*)L.x, L.y, 1, nullptr, nullptr, nullptr);
                go(k_rb_half<T>, blocks_for(L.n), kThreads, 0, L, (const T*)L.y, L.x, 0, nullptr, nullptr, nullptr);
                go(k_rb_half<T>, blocks_for(L.n), kThreads, 0, L, (const T*)L.x, L.y, 1, nullptr, nullptr, nullptr);
                go(k_rb_half<T>, blocks_for(L.n), kThreads, 0, L, (const T*)L.y, L.x, 0, fpartial_.p,
                   counters_.p + kPostMean, mo);
                launches_ += 5;
            }
            continue;
        }
        go(k_post1<T>, blocks_for(L.n), kThreads, 0, L);
        const bool want_mean = (l == 0) && L.singular;
        go(k_post2<T, Epi>, blocks_for(L.n), kThreads, 0, L, fpartial_.p, counters_.p + kPostMean,
           want_mean ? mean_out : nullptr, epi);
        launches_ += 3;
    }
    if (!V[0].singular) TPA_CUDA(cudaMemsetAsync(mean_out, 0, sizeof(double), stream_));
    TPA_CUDA(cudaGetLastError());
}

template void DeviceSolver::enqueue_vcycle<double>(const double*, const double*, double*);
template void DeviceSolver::enqueue_vcycle<float>(const double*, const double*, double*);

void DeviceSolver::vcycle_fused(const double* r, double* z, int precision) {
    const Launch go{stream_, pdl_};
    const int n = levels_[0].n;
    const int nl = int(levels_.size());
    double* rsum = lsum_.p;  // slot 0: level-0 RHS sum
    double* mean = lsum_.p + nl;
    go(k_sum_into, fold_grid(k_sum_into, kThreads, blocks_for(n), kMaxGrid), kThreads, 0, n, r, fpartial_.p,
       counters_.p + kRsum, rsum);
    ++launches_;
    if (precision == 0) enqueue_vcycle<double>(r, rsum, mean);
    else enqueue_vcycle<float>(r, rsum, mean);
    go(k_z_out, blocks_for(n), kThreads, 0, n, precision ? vf_[0].x : nullptr,
                                                      precision ? nullptr : vd_[0].x, mean, z);
    ++launches_;
    TPA_CUDA(cudaGetLastError());
}

// One CG iteration: the direction p = z + beta p (from the previous V-cycle)
// with Ap and alpha, the x / r update, the V-cycle, r'z and the stopping rules
// (which set the loop condition when `set_cond`).
void DeviceSolver::enqueue_cg_body(int precision, cudaGraphConditionalHandle handle, int set_cond) {
    const Launch go{stream_, pdl_};
    const int n = levels_[0].n;
    const int nl = int(levels_.size());
    CgState* s = reinterpret_cast<CgState*>(cgs_.p);
    double* mean = lsum_.p + nl;
    const LevelView<double>& A = vd_[0];
    const DevLevel& L0 = levels_[0];
    // xv: the V-cycle's finest-level output (z = xv - mean); r, the ping-pong
    // pair (pa, pb) of search directions and ap in the storage type P
    auto body = [&](auto* xv, auto* r, auto* pa, auto* pb, auto* ap) {
        using T = std::remove_pointer_t<decltype(xv)>;
        using P = std::remove_pointer_t<decltype(r)>;
        // z = M r and r'z (beta, or the start of a run)
        if (std::is_same<P, double>::value && rz_foldable()) {
            // r'z in the V-cycle's last kernel
            const CgRz epi{r_.p, fpartial2_.p, s};
            enqueue_vcycle_epi<T>(r_.p, &s->rsum, mean, epi);
        } else {
            enqueue_vcycle<T>((const P*)r, &s->rsum, mean);
            go(k_cg_z<T, P>, fold_grid(k_cg_z<T, P>, kThreads, blocks_for((n + 3) / 4), kMaxGrid), kThreads, 0, n,
               (const T*)xv, mean, (const P*)r, fpartial_.p, counters_.p + kCgZ, s);
        }
        // p = z + beta p_old, Ap and alpha = gamma / p'Ap
        if (sdev_[0].vec && tdev_.size() && tdev_[0].stream) {
            const StreamGeom g = stream_cg_geom();
            with_cg_rows(g.rows, [&](auto rows) {
                constexpr int RW = decltype(rows)::value;
                go(v_stream_dir_ap<T, P, RW>, tdev_[0].cg_grid, kStreamWarps * 32, 0, sd_[0], g, (const T*)xv, mean,
                   pa, pb, ap, fpartial_.p, counters_.p + kCgAp, s);
            });
        } else if (sdev_[0].vec)
            go(v_cg_dir_ap<T, P>, fold_grid(v_cg_dir_ap<T, P>, 256, (sd_[0].nblocks + 3) / 4, kMaxGrid), 256, 0,
               sd_[0], (const T*)xv, mean, pa, pb, ap, fpartial_.p, counters_.p + kCgAp, s);
        else if (sdev_[0].on)
            with_nxc(sd_[0], [&](auto nxc) {
                constexpr int N = decltype(nxc)::value;
                go(s_cg_dir_ap<T, P, N>, fold_grid(s_cg_dir_ap<T, P, N>, sd_[0].cpb, sd_[0].nblocks, kMaxGrid),
                   sd_[0].cpb, 0, sd_[0], (const T*)xv, mean, pa, pb, ap, fpartial_.p, counters_.p + kCgAp, s);
            });
        else
            go(k_cg_dir_ap<T, P>, fold_grid(k_cg_dir_ap<T, P>, kThreads, blocks_for(n), kMaxGrid), kThreads, 0, A,
               (const T*)xv, mean, pa, pb, ap, fpartial_.p, counters_.p + kCgAp, s);
        // x, r, the callback and the loop condition
        go(k_cg_update<P>, fold_grid(k_cg_update<P>, kThreads, blocks_for(n), kMaxGrid), kThreads, 0, n, xw_.p, r, pa,
           pb, (const P*)ap, L0.const_vol ? nullptr : A.vol, L0.vol0, fpartial_.p, fpartial2_.p,
           counters_.p + kCgUpdate, s, handle, set_cond);
    };
    if (precision == 0) {
        body(vd_[0].x, r_.p, p_.p, z_.p, ap_.p);
    } else if (precision == 1) {
        body(vf_[0].x, r_.p, p_.p, z_.p, ap_.p);
    } else {
        // the refinement solve's inner runs: FP32 r, directions and Ap
        float* w = ir_.p;
        const size_t n4 = ir_stride();
        body(vf_[0].x, w, w + n4, w + 2 * n4, w + 3 * n4);
    }
    TPA_CUDA(cudaGetLastError());
}

// The finest level is a CSR level swept by the multi-CTA kernels (not the tail
// or the cooperative cycle), with the damped-Jacobi post-smoothing, and is
// singular (its last post-smoothing folds the mean): r'z can ride on that fold.
// The structured and vectorized post-smoothings can carry it too (s_post2,
// v_sweep take the epilogue), but their folding grids are capped and stride
// over the level.  On the vectorized 2048^2 level the extra r stream cost more
// than the separate pass it replaces (3.35 -> 3.38 ms), and the structured
// kernel, with the same capped grid, is left out with it.  The CSR
// post-smoothing has one thread per cell and gains (droplet: 2.56 -> 2.49 ms).
// The row-streamed finest level (v_stream_up) takes the epilogue as well, but
// its r loads raised the kernel from 21.6 to 34-35 µs on 2048^2, plain or
// staged by cp.async, about what the separate pass costs (12.8 µs); it is left
// out too.
bool DeviceSolver::rz_foldable() const {
    return tail_first_ > 0 && coop_grid_ == 0 && !rb_ && levels_[0].ncomp == 1 && !sdev_.empty() && !sdev_[0].on;
}

cudaGraphExec_t DeviceSolver::cg_graph(int precision) {
    if (cg_exec_[precision]) return cg_exec_[precision];
    cudaGraph_t g;
    TPA_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle handle;
    TPA_CUDA(cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault));
    alignas(cudaGraphNodeParams) unsigned char cp_storage[sizeof(cudaGraphNodeParams)];
    std::memset(cp_storage, 0, sizeof(cp_storage));
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_storage);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    TPA_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    cudaStream_t saved = stream_;
    stream_ = own_stream_;
    const int saved_launches = launches_;
    TPA_CUDA(cudaStreamBeginCaptureToGraph(stream_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_cg_body(precision, handle, 1);
    cudaGraph_t captured;
    cudaError_t ce = cudaStreamEndCapture(stream_, &captured);
    stream_ = saved;
    // + direction/Ap, update and (unless folded) z
    graph_body_launches_[precision] = launches_ - saved_launches + (precision < 2 && rz_foldable() ? 2 : 3);
    launches_ = saved_launches;
    if (ce != cudaSuccess) {
        cudaGraphDestroy(g);
        throw Error(2, std::string("graph capture failed: ") + cudaGetErrorString(ce));
    }
    cudaGraphExec_t exec;
    cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) throw Error(2, std::string("graph instantiation failed: ") + cudaGetErrorString(ie));
    cg_exec_[precision] = exec;
    return exec;
}

void DeviceSolver::cg_fused(int precision, double target, int itmax, int& niter, int& flags) {
    const int n = levels_[0].n;
    const Launch go{stream_, pdl_};
    CgState* s = reinterpret_cast<CgState*>(cgs_.p);
    if (precision == 2) {
        if (coop_grid_ > 0) throw Error(5, "the refinement solve runs the multi-launch V-cycle, not the cooperative one");
        if (ir_.n != 4 * ir_stride()) {
            destroy_graphs();  // a captured body holds the old addresses
            ir_.alloc(4 * ir_stride());
            TPA_CUDA(cudaMemsetAsync(ir_.p, 0, ir_.n * sizeof(float), stream_));
        }
    }
    cudaGraphExec_t exec = cg_graph(precision);
    // a run: the state, r = b - A x and sum(r); the loop bodies follow
    go(k_cg_set, 1, 1, 0, s, target, itmax);
    if (precision == 2)
        // an inner run of the refinement solve starts from the true residual
        go(k_ir_start, fold_grid(k_ir_start, kThreads, blocks_for(n), kMaxGrid), kThreads, 0, n, (const double*)r_.p,
           ir_.p, fpartial_.p, counters_.p + kCgRes, s);
    else if (sdev_[0].vec)
        go(v_cg_residual, fold_grid(v_cg_residual, 256, (sd_[0].nblocks + 3) / 4, kMaxGrid), 256, 0, sd_[0], b_.p, xw_.p, r_.p,
           fpartial_.p, counters_.p + kCgRes, s);
    else if (sdev_[0].on)
        with_nxc(sd_[0], [&](auto nxc) {
            constexpr int N = decltype(nxc)::value;
            go(s_cg_residual<N>, fold_grid(s_cg_residual<N>, sd_[0].cpb, sd_[0].nblocks, kMaxGrid), sd_[0].cpb, 0, 
                sd_[0], b_.p, xw_.p, r_.p, fpartial_.p, counters_.p + kCgRes, s);
        });
    else
        go(k_cg_residual, fold_grid(k_cg_residual, kThreads, blocks_for(n), kMaxGrid), kThreads, 0, vd_[0], b_.p, xw_.p, r_.p, fpartial_.p,
                                                                counters_.p + kCgRes, s);
    launches_ += 2;
    CgState hs;
    std::memset(&hs, 0, sizeof(hs));
    if (itmax > 0 && std::getenv("TPAGMG_NO_GRAPH")) {
        // the same iteration launched kernel by kernel, stopping rules read on
        // the host after each one (profiling and diagnosis)
        bool stop = false;
        while (!stop) {
            const int before = launches_;
            enqueue_cg_body(precision, cudaGraphConditionalHandle(), 0);
            launches_ = before + graph_body_launches_[precision];
            TPA_CUDA(cudaMemcpyAsync(&hs, s, sizeof(CgState), cudaMemcpyDeviceToHost, stream_));
            TPA_CUDA(cudaStreamSynchronize(stream_));
            stop = (hs.flags & (kCgHalt | 1)) || hs.iter >= hs.itmax;
        }
    } else if (itmax > 0) {
        TPA_CUDA(cudaGraphLaunch(exec, stream_));
        TPA_CUDA(cudaMemcpyAsync(&hs, s, sizeof(CgState), cudaMemcpyDeviceToHost, stream_));
        TPA_CUDA(cudaStreamSynchronize(stream_));
        // every body ran its kernels; a body that halted is not counted
        const int bodies = hs.iter + ((hs.flags & kCgHalt) ? 1 : 0);
        launches_ += bodies * graph_body_launches_[precision];
    }
    TPA_CUDA(cudaGetLastError());
    niter = hs.iter;
    flags = hs.flags;
}

double DeviceSolver::time_fused(int which, int level, int precision, int iters) {
    if (level < 0 || level >= tail_first_) throw Error(1, "level is handled by the single-CTA tail");
    cudaEvent_t e0, e1;
    TPA_CUDA(cudaEventCreate(&e0));
    TPA_CUDA(cudaEventCreate(&e1));
    auto one = [&](const auto& V, auto tag) {
        using T = decltype(tag);
        const LevelView<T>& L = V[size_t(level)];
        switch (which) {
            case 0: k_post2<T><<<blocks_for(L.n), kThreads, 0, stream_>>>(L, fpartial_.p, counters_.p, nullptr); break;
            case 1:
                k_restrict<T><<<blocks_for(4 * int64_t(L.nc)), kThreads, 0, stream_>>>(L, V[size_t(level + 1)].b,
                                                                                        fpartial_.p, counters_.p,
                                                                                        nullptr);
                break;
            case 2: k_prolong<T><<<blocks_for(L.n), kThreads, 0, stream_>>>(L, V[size_t(level + 1)].x); break;
            case 4: k_pre2<T, T><<<blocks_for(L.n), kThreads, 0, stream_>>>(L, L.b, nullptr); break;
            case 5: k_residual<T><<<blocks_for(L.n), kThreads, 0, stream_>>>(L); break;
            default: throw Error(1, "unknown kernel");
        }
    };
    auto one_s = [&](const auto& S, auto tag) {
        using T = decltype(tag);
        const SView<T>& L = S[size_t(level)];
        const int g = L.nblocks, th = L.cpb;
        T* bc = sizeof(T) == 8 ? (T*)vd_[size_t(level + 1)].b : (T*)vf_[size_t(level + 1)].b;
        const T* xc = sizeof(T) == 8 ? (const T*)vd_[size_t(level + 1)].x : (const T*)vf_[size_t(level + 1)].x;
        if (sdev_[size_t(level)].vec) {
            const int groups = (L.nblocks + 3) / 4;
            switch (which) {
                case 0: v_sweep<T, false><<<groups, 256, 0, stream_>>>(L, L.y, L.x, nullptr, nullptr, nullptr); break;
                case 1: v_restrict<T><<<groups, 256, 0, stream_>>>(L, bc, fpartial_.p, counters_.p, nullptr); break;
                case 2: v_prolong<T><<<groups, 256, 0, stream_>>>(L, xc); break;
                case 4: v_pre2<T, T><<<groups, 256, 0, stream_>>>(L, L.b, nullptr); break;
                case 5: v_residual<T><<<groups, 256, 0, stream_>>>(L); break;
                default: throw Error(1, "unknown kernel");
            }
            return;
        }
        with_nxc(L, [&](auto nxc) {
            constexpr int N = decltype(nxc)::value;
            switch (which) {
                case 0: s_post2<T, N><<<g, th, 0, stream_>>>(L, fpartial_.p, counters_.p, nullptr); break;
                case 1: s_restrict<T, N><<<g, th, th * sizeof(T), stream_>>>(L, bc, fpartial_.p, counters_.p, nullptr); break;
                case 2: s_prolong<T, N><<<g, th, 0, stream_>>>(L, xc); break;
                case 4: s_pre2<T, T, N><<<g, th, 0, stream_>>>(L, L.b, nullptr); break;
                case 5: s_residual<T, N><<<g, th, 0, stream_>>>(L); break;
                default: throw Error(1, "unknown kernel");
            }
        });
    };
    // 6 / 7: the down / up tile kernel of a tiled CSR level
    auto one_tile = [&](const auto& V, auto tag) {
        using T = decltype(tag);
        const TileDev& D = tdev_[size_t(level)];
        const LevelView<T>& L = V[size_t(level)];
        const TileView<T>& TV = tile_view<T>(level);
        with_tile_threads(D.nt, [&](auto nt) {
            constexpr int NT = decltype(nt)::value;
            const size_t sm = tile_down_smem<T>(D.n3max, D.n2max, D.n1max, D.emax);
            if (which == 6 && level == 0)  // the finest level reads the FP64 residual, as in the cycle
                k_tile_down<T, double, NT><<<D.ntiles, NT, sm, stream_>>>(
                    L, TV, (const double*)r_.p, nullptr, V[size_t(level + 1)].b, fpartial_.p, counters_.p, nullptr);
            else if (which == 6)
                k_tile_down<T, T, NT><<<D.ntiles, NT, sm, stream_>>>(L, TV, (const T*)L.b, nullptr,
                                                                     V[size_t(level + 1)].b, fpartial_.p,
                                                                     counters_.p, nullptr);
            else
                k_tile_up<T, MeanOnly, NT><<<D.ntiles, NT, tile_up_smem<T>(D.n3max, D.n2max, D.n1max, D.emax),
                                            stream_>>>(L, TV, (const T*)V[size_t(level + 1)].x, fpartial_.p,
                                                       counters_.p, nullptr, MeanOnly());
        });
    };
    // 8 / 9: the down / up row-streaming kernel of a streamed lattice level
    auto one_stream = [&](const auto& S, const auto& V, auto tag) {
        using T = decltype(tag);
        constexpr bool fp32 = std::is_same<T, float>::value;
        const SView<T>& L = S[size_t(level)];
        const StreamGeom g = stream_geom(level, fp32);
        const int grid = tdev_[size_t(level)].sgrid[fp32 ? 1 : 0];
        with_stream_rows(g.rows, [&](auto rows) {
            constexpr int RW = decltype(rows)::value;
            if (which == 8 && level == 0)  // the finest level reads the FP64 residual, as in the cycle
                v_stream_down<T, double, RW><<<grid, kStreamWarps * 32, 0, stream_>>>(
                    L, g, (const double*)r_.p, nullptr, V[size_t(level + 1)].b, fpartial_.p, counters_.p, nullptr);
            else if (which == 8)
                v_stream_down<T, T, RW><<<grid, kStreamWarps * 32, 0, stream_>>>(
                    L, g, (const T*)L.b, nullptr, V[size_t(level + 1)].b, fpartial_.p, counters_.p, nullptr);
            else
                v_stream_up<T, MeanOnly, RW><<<grid, kStreamWarps * 32, 0, stream_>>>(
                    L, g, (const T*)V[size_t(level + 1)].x, fpartial_.p, counters_.p, nullptr, MeanOnly());
        });
    };
    auto launch = [&]() {
        if (which == 8 || which == 9) {
            if (size_t(level) >= tdev_.size() || !tdev_[size_t(level)].stream)
                throw Error(1, "level does not run on the row-streaming kernels");
            if (precision == 0) one_stream(sd_, vd_, double(0));
            else one_stream(sf_, vf_, float(0));
            return;
        }
        if (which == 6 || which == 7) {
            if (size_t(level) >= tdev_.size() || !tdev_[size_t(level)].on)
                throw Error(1, "level does not run on CSR tiles");
            if (precision == 0) one_tile(vd_, double(0));
            else one_tile(vf_, float(0));
            return;
        }
        if (which == 3) {
            if (precision != 0 || level != 0) throw Error(1, "the CG operator runs in FP64 on the finest level");
            CgState* s = reinterpret_cast<CgState*>(cgs_.p);
            if (sdev_[0].vec)
                v_cg_ap<<<fold_grid(v_cg_ap, 256, (sd_[0].nblocks + 3) / 4, kMaxGrid), 256, 0, stream_>>>(sd_[0], p_.p, ap_.p,
                                                                                          fpartial_.p,
                                                                                          counters_.p + kCgAp, s);
            else if (sdev_[0].on)
                with_nxc(sd_[0], [&](auto nxc) {
                    constexpr int N = decltype(nxc)::value;
                    s_cg_ap<N><<<fold_grid(s_cg_ap<N>, sd_[0].cpb, sd_[0].nblocks, kMaxGrid), sd_[0].cpb, 0, stream_>>>(
                        sd_[0], p_.p, ap_.p, fpartial_.p, counters_.p + kCgAp, s);
                });
            else
                k_cg_ap<<<fold_grid(k_cg_ap, kThreads, blocks_for(vd_[0].n), kMaxGrid), kThreads, 0, stream_>>>(vd_[0], p_.p, ap_.p, fpartial_.p,
                                                                         counters_.p + kCgAp, s);
        } else if (sdev_[size_t(level)].on) {
            if (precision == 0) one_s(sd_, double(0));
            else one_s(sf_, float(0));
        } else if (precision == 0) {
            one(vd_, double(0));
        } else {
            one(vf_, float(0));
        }
    };
    launch();
    TPA_CUDA(cudaEventRecord(e0, stream_));
    for (int k = 0; k < iters; ++k) launch();
    TPA_CUDA(cudaEventRecord(e1, stream_));
    TPA_CUDA(cudaEventSynchronize(e1));
    TPA_CUDA(cudaGetLastError());
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return double(ms) / iters;
}

}  // namespace tpa

namespace tpa {

template <typename T>
const TileView<T>& DeviceSolver::tile_view(int l) const {
    if constexpr (std::is_same<T, double>::value) return td_[size_t(l)];
    else return tf_[size_t(l)];
}

template <typename T, typename TB>
static void allow_tile_down_smem(size_t bytes) {
    TPA_CUDA(cudaFuncSetAttribute(k_tile_down<T, TB, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    TPA_CUDA(cudaFuncSetAttribute(k_tile_down<T, TB, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    TPA_CUDA(cudaFuncSetAttribute(k_tile_down<T, TB, 1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
}
template <typename T, typename Epi>
static void allow_tile_up_smem(size_t bytes) {
    TPA_CUDA(cudaFuncSetAttribute(k_tile_up<T, Epi, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    TPA_CUDA(cudaFuncSetAttribute(k_tile_up<T, Epi, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    TPA_CUDA(cudaFuncSetAttribute(k_tile_up<T, Epi, 1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
}

// Tiles of every CSR level of the multi-CTA part of the default cycle (not the
// stencil levels, the tail, the red-black smoother or the cooperative cycle).
void DeviceSolver::upload_tiles(const Hierarchy& h) {
    const int nl = int(levels_.size());
    const TuneConfig cfg = effective_tuning();
    tdev_.clear();
    tdev_.resize(size_t(nl));
    td_.assign(size_t(nl), TileView<double>{});
    tf_.assign(size_t(nl), TileView<float>{});
    if (!cfg.tiles || rb_ || !fused_ok_ || coop_grid_ > 0) return;
    // a tile's arrays live in shared memory: at most this many cells (rings <= 3)
    int sms = 148;
    TPA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
    size_t down_d = 0, up_d = 0;
    for (int l = 0; l < tail_first_ && l + 1 < nl; ++l) {
        if (sdev_[size_t(l)].vec) {  // stencil tiles and row streaming need no lists
            const bool small = levels_[size_t(l)].n <= kStencilTileCells;
            TileDev& D = tdev_[size_t(l)];
            D.stream = sdev_[size_t(l)].snbx > 0 && (cfg.tiles == 5 || (cfg.tiles == 4 && !small));
            D.vec = !D.stream && (cfg.tiles == 2 || (cfg.tiles >= 3 && small));
            if (D.stream)
                for (int fp32 = 0; fp32 < 2; ++fp32) {
                    const int ctas = fp32 ? stream_ctas_per_sm<float>() : stream_ctas_per_sm<double>();
                    D.srows[fp32] = stream_rows(sdev_[size_t(l)].snbx, sdev_[size_t(l)].snby, sms, ctas);
                    const StreamGeom g = stream_geom(l, fp32 != 0);
                    D.sgrid[fp32] = int(std::min<int64_t>((int64_t(g.nsx) * g.nsy + kStreamWarps - 1) / kStreamWarps,
                                                          int64_t(ctas) * sms));
                }
            if (D.stream && l == 0) {  // the CG's direction and operator product on the finest level
                D.cg_rows = stream_rows(sdev_[0].snbx, sdev_[0].snby, sms, kStreamCgCtas, kStreamCgCols, 2, false);
                const StreamGeom g = stream_cg_geom();
                D.cg_grid = int(std::min<int64_t>((int64_t(g.nsx) * g.nsy + kStreamWarps - 1) / kStreamWarps,
                                                  int64_t(kStreamCgCtas) * sms));
            }
            continue;
        }
        if (sdev_[size_t(l)].on) continue;
        const HostLevel& hl = h.levels[size_t(l)];
        const TileLevelHost T = build_tiles(hl.op.A, hl.op.mesh.nblocks(), hl.op.mesh.cells_per_block(), hl.owner,
                                            h.levels[size_t(l + 1)].op.A.n, kTileMaxCells);
        if (!T.ok) continue;
        TileDev& D = tdev_[size_t(l)];
        D.ntiles = T.ntiles;
        D.n3max = T.n3max;
        D.n2max = T.n2max;
        D.n1max = T.n1max;
        D.emax = T.emax;
        // 2 CTAs of 1024 threads, 4 of 512 fit an SM (by threads)
        D.nt = T.ntiles <= 2 * sms ? 1024 : T.ntiles <= 4 * sms ? 512 : 256;
        D.nent = int(T.pos.size());
        D.cell.upload(T.cell.data(), T.cell.size(), stream_);
        D.own.upload(T.own.data(), T.own.size(), stream_);
        D.cell_off.upload(T.cell_off.data(), T.cell_off.size(), stream_);
        D.ring.upload(T.ring.data(), T.ring.size(), stream_);
        D.lrp.upload(T.lrp.data(), T.lrp.size(), stream_);
        D.lrp_off.upload(T.lrp_off.data(), T.lrp_off.size(), stream_);
        D.ent_off.upload(T.ent_off.data(), T.ent_off.size(), stream_);
        D.pos.upload(T.pos.data(), T.pos.size(), stream_);
        D.lcol.upload(T.lcol.data(), T.lcol.size(), stream_);
        D.co.upload(T.co.data(), T.co.size(), stream_);
        D.co_off.upload(T.co_off.data(), T.co_off.size(), stream_);
        D.ch.upload(T.ch.data(), T.ch.size(), stream_);
        D.val_d.alloc(T.pos.size());
        D.val_f.alloc(T.pos.size());
        TPA_CUDA(cudaStreamSynchronize(stream_));  // the host arrays go out of scope
        auto fill = [&](auto& v, auto* val) {
            v.ntiles = D.ntiles;
            v.n3max = D.n3max;
            v.n2max = D.n2max;
            v.n1max = D.n1max;
            v.emax = D.emax;
            v.cell = D.cell.p;
            v.own = D.own.p;
            v.cell_off = D.cell_off.p;
            v.ring = reinterpret_cast<const int4*>(D.ring.p);
            v.lrp = D.lrp.p;
            v.lrp_off = D.lrp_off.p;
            v.ent_off = D.ent_off.p;
            v.val = val;
            v.lcol = reinterpret_cast<const short*>(D.lcol.p);
            v.co = D.co.p;
            v.co_off = D.co_off.p;
            v.ch = reinterpret_cast<const short4*>(D.ch.p);
        };
        fill(td_[size_t(l)], D.val_d.p);
        fill(tf_[size_t(l)], D.val_f.p);
        down_d = std::max(down_d, tile_down_smem<double>(D.n3max, D.n2max, D.n1max, D.emax));
        up_d = std::max(up_d, tile_up_smem<double>(D.n3max, D.n2max, D.n1max, D.emax));
        D.on = true;
    }
    if (down_d == 0) return;
    // one partial sum per tile in the folds of the tile kernels
    size_t ntiles = 0;
    for (const auto& D : tdev_) ntiles = std::max(ntiles, size_t(D.on ? D.ntiles : 0));
    if (ntiles > fpartial_.n) {
        fpartial_.alloc(ntiles);
        fpartial2_.alloc(ntiles);
    }
    int optin = 0;
    TPA_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_));
    if (down_d > size_t(optin) || up_d > size_t(optin)) {
        for (auto& D : tdev_) D.on = false;
        return;
    }
    allow_tile_down_smem<double, double>(down_d);
    allow_tile_down_smem<float, double>(down_d);
    allow_tile_down_smem<float, float>(down_d);
    allow_tile_up_smem<double, MeanOnly>(up_d);
    allow_tile_up_smem<float, MeanOnly>(up_d);
    allow_tile_up_smem<double, CgRz>(up_d);
    allow_tile_up_smem<float, CgRz>(up_d);
    gather_tile_values();
    destroy_graphs();
}

void DeviceSolver::gather_tile_values() {
    for (size_t l = 0; l < tdev_.size(); ++l) {
        TileDev& D = tdev_[l];
        if (!D.on || D.nent == 0) continue;
        const DevLevel& L = levels_[l];
        const int g = int(std::min<int64_t>((D.nent + kThreads - 1) / kThreads, kMaxGrid));
        k_tile_gather<double><<<g, kThreads, 0, stream_>>>(D.nent, D.pos.p, L.d.val.p, D.val_d.p);
        k_tile_gather<float><<<g, kThreads, 0, stream_>>>(D.nent, D.pos.p, L.f.val.p, D.val_f.p);
    }
    TPA_CUDA(cudaGetLastError());
    TPA_CUDA(cudaStreamSynchronize(stream_));
}

int DeviceSolver::streamed_levels() const {
    int k = 0;
    for (const auto& d : tdev_) k += d.stream ? 1 : 0;
    return k;
}

int DeviceSolver::tiled_levels() const {
    int k = 0;
    for (const auto& d : tdev_) k += (d.on || d.vec || d.stream) ? 1 : 0;
    return k;
}

StreamGeom DeviceSolver::stream_cg_geom() const {
    const StructDev& D = sdev_[0];
    StreamGeom g;
    g.nbx = D.snbx;
    g.nby = D.snby;
    g.rows = tdev_[0].cg_rows;
    g.nsx = (16 * D.snbx + kStreamCgCols - 1) / kStreamCgCols;
    g.nsy = (16 * D.snby + g.rows - 1) / g.rows;
    return g;
}

// The block lattice of a level for the row-streaming kernels (stream.cuh):
// returns its width nbx in blocks (height in `nby`), or 0 when the level does not
// qualify.  It qualifies when both axes are periodic and its 16 x 16 blocks are
// one tree level filling an nbx x nby rectangle in row-major order (the
// (level, j, i) sort), with the same-size neighbours of the periodic lattice.
// The next level must be the lattice halved in both directions: block map with
// coarse block (j / 2) (nbx / 2) + i / 2, offsets 8 (i mod 2) and 8 (j mod 2),
// scale 2.
static int stream_lattice(const Mesh& m, const Mesh& mc, const StructLevel& st, int& nby) {
    nby = 0;
    if (!m.periodic[0] || !m.periodic[1] || m.bs[0] != 16 || m.bs[1] != 16 || m.keys.empty()) return 0;
    const int lev = key_level(m.keys[0]);
    int64_t nbx = 0, ny = 0;
    for (uint64_t k : m.keys) {
        if (key_level(k) != lev) return 0;
        nbx = std::max<int64_t>(nbx, key_i(k) + 1);
        ny = std::max<int64_t>(ny, key_j(k) + 1);
    }
    const int64_t nb = m.nblocks();
    if (nbx * ny != nb || nbx < 2 || ny < 2 || nbx % 2 || ny % 2 || nb * 256 > int64_t(INT32_MAX)) return 0;
    if (mc.nblocks() * 4 != nb || int64_t(st.nbr.size()) != 4 * nb || int64_t(st.map.size()) != 4 * nb) return 0;
    for (int64_t b = 0; b < nb; ++b) {
        const int64_t i = b % nbx, j = b / nbx;
        if (m.keys[size_t(b)] != pack_key(lev, i, j)) return 0;
        const int32_t* q = &st.nbr[size_t(4 * b)];
        if (q[0] != j * nbx + (i + nbx - 1) % nbx || q[1] != j * nbx + (i + 1) % nbx ||
            q[2] != ((j + ny - 1) % ny) * nbx + i || q[3] != ((j + 1) % ny) * nbx + i)
            return 0;
        const int32_t* mp = &st.map[size_t(4 * b)];
        if (mp[0] != (j / 2) * (nbx / 2) + i / 2 || mp[1] != (i % 2) * 8 || mp[2] != (j % 2) * 8 || mp[3] != 2) return 0;
    }
    nby = int(ny);
    return int(nbx);
}

StreamGeom DeviceSolver::stream_geom(int l, bool fp32) const {
    const StructDev& D = sdev_[size_t(l)];
    StreamGeom g;
    g.nbx = D.snbx;
    g.nby = D.snby;
    g.rows = tdev_[size_t(l)].srows[fp32 ? 1 : 0];
    g.nsx = (16 * D.snbx + kStreamCols - 1) / kStreamCols;
    g.nsy = (16 * D.snby + g.rows - 1) / g.rows;
    return g;
}

// Block-structured copies of every level that qualifies: 16x16-style blocks
// (32 to 1024 cells, a multiple of 32), a valid block map of the transfer and
// the transfer's inverse diagonal equal to the smoother's.
void DeviceSolver::upload_structured(const Hierarchy& h) {
    const int nl = int(levels_.size());
    rl_ready_ = false;  // the device refresh gathers into the stencil copies made here
    sdev_.clear();
    sdev_.resize(size_t(nl));
    sd_.assign(size_t(nl), SView<double>{});
    sf_.assign(size_t(nl), SView<float>{});
    const TuneConfig cfg = effective_tuning();
    const bool disabled = cfg.structured == 0;
    for (int l = 0; l < nl; ++l) {
        const HostLevel& hl = h.levels[size_t(l)];
        const int cpb = hl.op.mesh.bs[0] * hl.op.mesh.bs[1];
        // a stencil row is c0 (count x_c - neighbours): not a row with an
        // open-face conductance on its diagonal
        const bool open_diag = std::any_of(hl.op.bdiag.begin(), hl.op.bdiag.end(), [](double v) { return v != 0.0; });
        if (disabled || open_diag || l >= tail_first_ || l + 1 >= nl || cpb < 32 || cpb > 1024 || cpb % 32) continue;
        StructLevel st = build_struct(hl, &h.levels[size_t(l + 1)].op.mesh);
        if (!st.has_map || !st.tinv_same) continue;
        // Variable-coefficient levels with coarse-fine exception rows are small and
        // latency-bound; the CSR kernels (one index chain per row, no divergence
        // between stencil and exception rows) are faster there.  Structured mode 2
        // (TPAGMG_STRUCTURED=all, or the autotuner) uses the stencil path on every
        // level that has a block map.
        if (cfg.structured < 2 && !(st.const_coef && st.nex == 0)) continue;
        StructDev& D = sdev_[size_t(l)];
        D.on = true;
        D.vec = st.const_coef && st.nex == 0 && st.nx == 16 && st.ny == 16 && cfg.vectorized;
        D.nex = st.nex;
        D.const_coef = st.const_coef;
        D.const_diag = st.const_diag;
        D.nbr.upload(st.nbr.data(), st.nbr.size(), stream_);
        D.map.upload(st.map.data(), st.map.size(), stream_);
        std::vector<float> f;
        if (!st.const_coef) {
            D.cx_d.upload(st.cx.data(), st.cx.size(), stream_);
            D.cy_d.upload(st.cy.data(), st.cy.size(), stream_);
            f.assign(st.cx.begin(), st.cx.end());
            D.cx_f.upload(f.data(), f.size(), stream_);
            std::vector<float> g(st.cy.begin(), st.cy.end());
            D.cy_f.upload(g.data(), g.size(), stream_);
            TPA_CUDA(cudaStreamSynchronize(stream_));
        }
        if (st.nex) {
            std::vector<int> ptr(st.ex_ptr.begin(), st.ex_ptr.end());
            D.ex.upload(st.ex.data(), st.ex.size(), stream_);
            D.ex_ptr.upload(ptr.data(), ptr.size(), stream_);
            D.ex_col.upload(st.ex_col.data(), st.ex_col.size(), stream_);
            D.exv_d.upload(st.ex_val.data(), st.ex_val.size(), stream_);
            std::vector<float> g(st.ex_val.begin(), st.ex_val.end());
            D.exv_f.upload(g.data(), g.size(), stream_);
            TPA_CUDA(cudaStreamSynchronize(stream_));
        }
        DevLevel& L = levels_[size_t(l)];
        const std::vector<double>& hv = hl.op.volumes;
        const bool const_vol = !hv.empty() && std::all_of(hv.begin(), hv.end(), [&](double v) { return v == hv[0]; });
        if (D.vec && st.const_diag && const_vol)
            D.snbx = stream_lattice(hl.op.mesh, h.levels[size_t(l + 1)].op.mesh, st, D.snby);
        auto fill = [&](auto& v, auto& DL, auto* cx, auto* cy, auto* exv, auto cast) {
            v.nx = hl.op.mesh.bs[0];
            v.ny = hl.op.mesh.bs[1];
            v.cpb = cpb;
            v.nblocks = int(hl.op.mesh.nblocks());
            v.n = L.n;
            v.nbr = D.nbr.p;
            v.cx = st.const_coef ? nullptr : cx;
            v.cy = st.const_coef ? nullptr : cy;
            v.c0 = cast(st.c0);
            v.dinv = st.const_diag ? nullptr : DL.dinv.p;
            v.dinv0 = cast(st.dinv.empty() ? 0.0 : st.dinv[0]);
            v.ex = st.nex ? D.ex.p : nullptr;
            v.ex_ptr = D.ex_ptr.p;
            v.ex_col = D.ex_col.p;
            v.ex_val = exv;
            v.map = D.map.p;
            v.vol = DL.vol.p;
            v.const_vol = const_vol ? 1 : 0;
            v.vol0 = cast(hl.op.volumes.empty() ? 0.0 : hl.op.volumes[0]);
            v.w = DL.w;
            v.tw = DL.tw;
            v.singular = L.ncomp == 1;
            v.cvol_inv = L.ncomp == 1 ? 1.0 / L.comp_volume[0] : 0.0;
            v.b = DL.b.p;
            v.bp = DL.bp.p;
            v.x = DL.x.p;
            v.y = DL.y.p;
            v.r = DL.r.p;
            v.s = DL.s.p;
            v.ccpb = cpb;
        };
        fill(sd_[size_t(l)], L.d, D.cx_d.p, D.cy_d.p, D.exv_d.p, [](double v) { return v; });
        fill(sf_[size_t(l)], L.f, D.cx_f.p, D.cy_f.p, D.exv_f.p, [](double v) { return float(v); });
    }
    // the cooperative V-cycle covers CSR levels only, one CTA of kTailThreads per SM
    coop_grid_ = 0;
    if (cfg.persistent && fused_ok_ && tail_ctas_ == 1) {
        bool csr = true;
        for (int l = 0; l < tail_first_; ++l) csr = csr && !sdev_[size_t(l)].on;
        int sms = 0, occ_f = 0, occ_d = 0;
        TPA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
        TPA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_f, k_vcycle_grid<float>, kTailThreads, 0));
        TPA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_d, k_vcycle_grid<double>, kTailThreads, 0));
        if (csr && occ_f >= 1 && occ_d >= 1) coop_grid_ = sms;
    }
    TPA_CUDA(cudaStreamSynchronize(stream_));
    destroy_graphs();
}

int DeviceSolver::structured_levels() const {
    int k = 0;
    for (const auto& d : sdev_) k += d.on ? 1 : 0;
    return k;
}

int64_t DeviceSolver::exception_rows() const {
    int64_t k = 0;
    for (const auto& d : sdev_) k += d.on ? d.nex : 0;
    return k;
}

}  // namespace tpa
