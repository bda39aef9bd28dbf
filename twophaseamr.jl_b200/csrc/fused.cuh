// Fused V-cycle and PCG kernels for the default cycle (two pre- and two
// post-sweeps, at most one ungauged component per level).
//
// Each kernel removes one or more grid-wide dependencies of the plain cycle of
// src/solvers/multigrid/cycles.jl:8-77 (ronaldremmerswaal/TwoPhaseAMR.jl):
//   k_pre2          both pre-sweeps from x = 0: the first sweep is pointwise,
//                   x1 = w D^-1 b, so the second one evaluates x1 at the
//                   neighbours on the fly; the RHS projection of the level
//                   (`_multigrid_project_component_rhs!`) is applied inline
//   k_residual, k_restrict  r = b - A x, s = Dt^-1 r, then b_c = P_tent.(r - wt A s)
//                   with the coarse RHS sum folded in the same launch
//   k_prolong       x += e - wt Dt^-1 A e with e = P_tent x_c, in place (it
//                   reads no neighbouring fine value)
//   k_tail          every level with at most kTailCells cells in one CTA
// Reductions fold their per-block partials in the last block to finish (a
// fixed-order fold: results do not depend on block scheduling).
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

namespace tpa {

// Levels at or below this many cells run in the coarse tail, one cluster of
// kTailCtasDefault CTAs of kTailThreads threads (TPAGMG_TAIL_CELLS, TPAGMG_TAIL_CTAS).
// Measured on the B200 (droplet AMR and uniform 2048^2 solves): the tail is bound
// by the latency of its dependent loads, so more CTAs or a larger tail (4096 to
// 32768 cells, 4 or 8 CTAs) were 2-15 % slower than 2048 cells in one CTA.
constexpr int kTailCellsDefault = 2048;
constexpr int kTailCtasDefault = 1;
constexpr int kTailThreads = 1024;

// First statement of every cycle kernel (programmatic dependent launch, sm_90
// and later): allow the next kernel of the stream to be scheduled now, then wait
// until the kernels this one depends on have completed and their writes are
// visible.  Nothing is read or written before the wait.  For a launch without
// the programmatic attribute both instructions return at once.
__device__ __forceinline__ void pdl_entry() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Pointers of one level in precision T, read by the fused kernels.
template <typename T>
struct LevelView {
    int n, nc;
    const int* rp;
    const int* ci;
    const T* val;
    const T* dinv;
    const T* tinv;
    const T* vol;
    const int* owner;
    const int* cptr;
    const int* child;
    T w, tw;
    int singular;      // ungauged component present (one)
    double cvol_inv;   // 1 / component volume
    T* b;              // restricted right-hand side (raw)
    T* bp;             // projected right-hand side
    T* x;              // iterate
    T* y;              // second iterate buffer
    T* r;              // residual
    T* s;              // Dt^-1 r
    const unsigned char* colour;  // red-black smoother (rb != 0): 0 red, 1 black
    int rb;
    T rbw;             // red-black half-sweep weight
    // open-face conductance per cell (finest level, FP64 view; null: no open
    // side).  The operator's diagonal holds it; the true-residual kernels, which
    // sum rows as a_ij (x_j - x_i), add it back as bdiag_i x_i.
    const double* bdiag;
};

// fold partial[0..count) in fixed order by one block; returns the sum in thread 0
__device__ __forceinline__ double fold_partials(const double* partial, int count) {
    __shared__ double sh[32];
    double acc = 0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) acc += ((volatile const double*)partial)[i];
    for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (!lane) sh[wid] = acc;
    __syncthreads();
    acc = 0;
    if (threadIdx.x < (blockDim.x >> 5)) acc = sh[threadIdx.x];
    if (wid == 0)
        for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    return acc;
}

__device__ __forceinline__ double fold_partials_max(const double* partial, int count) {
    __shared__ double sh[32];
    __shared__ int nan_seen;
    double m = 0;
    bool nan = false;
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        double q = ((volatile const double*)partial)[i];
        if (q != q) nan = true;
        m = fmax(m, q);
    }
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (threadIdx.x == 0) nan_seen = 0;
    if (!lane) sh[wid] = m;
    __syncthreads();
    if (nan) nan_seen = 1;
    m = 0;
    if (threadIdx.x < (blockDim.x >> 5)) m = sh[threadIdx.x];
    if (wid == 0)
        for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    __syncthreads();
    return nan_seen ? NAN : m;
}

__device__ __forceinline__ double block_sum_all(double v) {
    __shared__ double sh[32];
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (!lane) sh[wid] = v;
    __syncthreads();
    v = 0;
    if (threadIdx.x < (blockDim.x >> 5)) v = sh[threadIdx.x];
    if (wid == 0)
        for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Write this block's partial, and return true in the block that finishes last.
__device__ __forceinline__ bool publish_partial(double v, double* partial, unsigned* counter) {
    __shared__ bool last;
    v = block_sum_all(v);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = v;
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    return last;
}

// publish_partial of two block sums (v into p1, w into p2) under one counter
__device__ __forceinline__ bool publish_partial2(double v, double w, double* p1, double* p2, unsigned* counter) {
    __shared__ bool last;
    v = block_sum_all(v);
    w = block_sum_all(w);
    if (threadIdx.x == 0) {
        p1[blockIdx.x] = v;
        p2[blockIdx.x] = w;
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    return last;
}

// Epilogue of the finest level's last post-smoothing, which folds the volume
// mean of x: nothing more (MeanOnly), or -- inside the CG loop -- also the sum
// of r_i x_i, handed with the mean to the CG's own step (kRz), so that r'z of
// z = x - mean needs no pass of its own.
struct MeanOnly {
    static constexpr bool kRz = false;
    const double* r = nullptr;
    double* partial = nullptr;
    __device__ void operator()(double, double) const {}
};

// The last block folds sum V x (partial) and, with kRz, sum r x (epi.partial);
// thread 0 writes the mean and calls the epilogue.
template <typename Epi>
__device__ __forceinline__ void fold_mean(double v, double w, double* partial, unsigned* counter, double* mean_out,
                                          double cvol_inv, const Epi& epi) {
    if constexpr (Epi::kRz) {
        if (publish_partial2(v, w, partial, epi.partial, counter)) {
            const double s = fold_partials(partial, gridDim.x);
            const double rx = fold_partials(epi.partial, gridDim.x);
            if (threadIdx.x == 0) {
                const double mean = s * cvol_inv;
                *mean_out = mean;
                epi(mean, rx);
                *counter = 0;
            }
        }
    } else if (publish_partial(v, partial, counter)) {
        const double s = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            *mean_out = s * cvol_inv;
            *counter = 0;
        }
    }
}

template <typename T>
__device__ __forceinline__ T rowdot(const LevelView<T>& L, const T* v, int i) {
    T acc = T(0);
    for (int k = L.rp[i]; k < L.rp[i + 1]; ++k) acc += L.val[k] * v[L.ci[k]];
    return acc;
}

// ---------------------------------------------------------------------------------
// Per-level phases as device functions over a cell, shared by the multi-CTA
// kernels and the single-CTA tail.

// projected RHS value at cell j (in FP64 arithmetic)
template <typename T, typename TB>
__device__ __forceinline__ T proj_b(const LevelView<T>& L, const TB* b, double mean, int j) {
    double v = double(b[j]);
    if (L.singular) v -= double(L.vol[j]) * mean;
    return T(v);
}

template <typename T, typename TB>
__device__ __forceinline__ void pre2_cell(const LevelView<T>& L, const TB* b, double mean, int i) {
    T bi = proj_b<T, TB>(L, b, mean, i);
    T acc = T(0);
    for (int k = L.rp[i]; k < L.rp[i + 1]; ++k) {
        int j = L.ci[k];
        T bj = j == i ? bi : proj_b<T, TB>(L, b, mean, j);
        acc += L.val[k] * (L.w * L.dinv[j] * bj);
    }
    T x1 = L.w * L.dinv[i] * bi;
    L.x[i] = x1 + L.w * L.dinv[i] * (bi - acc);
    L.bp[i] = bi;
}

template <typename T>
__device__ __forceinline__ void residual_cell(const LevelView<T>& L, int i) {
    T ri = L.bp[i] - rowdot(L, L.x, i);
    L.r[i] = ri;
    L.s[i] = L.tinv[i] * ri;
}

// Restriction with four lanes per coarse cell (lane q takes children q, q + 4,
// ...; a coarse cell has one or four children): call from thread g = 4 J + q
// of a whole warp; returns the coarse value in every lane of the group, summed
// in the fixed order (c0 + c1) + (c2 + c3).
template <typename T>
__device__ __forceinline__ T restrict_quad(const LevelView<T>& L, int J, int q) {
    T acc = T(0);
    if (J < L.nc)
        for (int k = L.cptr[J] + q; k < L.cptr[J + 1]; k += 4) {
            const int i = L.child[k];
            acc += L.r[i] - L.tw * rowdot(L, L.s, i);
        }
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    return acc;
}

// x += e - wt Dt^-1 A e, e = xc[owner(.)]
template <typename T>
__device__ __forceinline__ void prolong_cell(const LevelView<T>& L, const T* xc, int i) {
    T ae = T(0);
    for (int k = L.rp[i]; k < L.rp[i + 1]; ++k) ae += L.val[k] * xc[L.owner[L.ci[k]]];
    L.x[i] += xc[L.owner[i]] - L.tw * L.tinv[i] * ae;
}

template <typename T>
__device__ __forceinline__ void sweep_cell(const LevelView<T>& L, const T* in, T* out, int i) {
    out[i] = in[i] + L.w * L.dinv[i] * (L.bp[i] - rowdot(L, in, i));
}

// Red-black Gauss-Seidel (an option; the reference smooths with damped
// Jacobi).  A half-sweep updates the cells of one colour from the iterate `in`
// and keeps the other colour, so that coupled cells of one colour (coarse-fine
// faces) read the values of the previous half-sweep.  Red then
// black before the coarse correction, the reverse after it: the V-cycle stays
// symmetric, as CG needs.

// first sweep from zero into `out`: red w D^-1 bp; black w D^-1 (bp - A x_red),
// the red values recomputed at the black cell's red neighbours
template <typename T, typename TB>
__device__ __forceinline__ void rb_first_cell(const LevelView<T>& L, const TB* b, double mean, T* out, int i) {
    const T bi = proj_b<T, TB>(L, b, mean, i);
    L.bp[i] = bi;
    if (L.colour[i] == 0) {
        out[i] = L.rbw * L.dinv[i] * bi;
        return;
    }
    T acc = T(0);
    for (int k = L.rp[i]; k < L.rp[i + 1]; ++k) {
        const int j = L.ci[k];
        if (L.colour[j] == 0) acc += L.val[k] * (L.rbw * L.dinv[j] * proj_b<T, TB>(L, b, mean, j));
    }
    out[i] = L.rbw * L.dinv[i] * (bi - acc);
}

// the half-sweep value of cell i of colour c from `in`
template <typename T>
__device__ __forceinline__ T rb_update(const LevelView<T>& L, const T* in, int i) {
    return in[i] + L.rbw * L.dinv[i] * (L.bp[i] - rowdot(L, in, i));
}

// two half-sweeps, colour c then the other, from `in` into `out` in one pass:
// a cell of the second colour recomputes its colour-c neighbours' first
// half-sweep values (the same arithmetic, so the same bits, as the
// half-sweep kernel writes); cells of one colour read only `in` values of
// their own colour, as in two separate half-sweeps
template <typename T>
__device__ __forceinline__ void rb_pair_cell(const LevelView<T>& L, const T* in, T* out, int c, int i) {
    if (L.colour[i] == c) {
        out[i] = rb_update(L, in, i);
        return;
    }
    T acc = T(0);
    for (int k = L.rp[i]; k < L.rp[i + 1]; ++k) {
        const int j = L.ci[k];
        acc += L.val[k] * (L.colour[j] == c ? rb_update(L, in, j) : in[j]);
    }
    out[i] = in[i] + L.rbw * L.dinv[i] * (L.bp[i] - acc);
}

// ---------------------------------------------------------------------------------
// multi-CTA kernels

// `level_sum` (may be null): the RHS sum of this level, folded by the kernel
// that produced b; mean = sum * cvol_inv.
template <typename T, typename TB>
__global__ void k_pre2(LevelView<T> L, const TB* __restrict__ b, const double* level_sum) {
    pdl_entry();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double mean = (L.singular && level_sum) ? *level_sum * L.cvol_inv : 0.0;
    if (i < L.n) pre2_cell<T, TB>(L, b, mean, i);
}

// one red-black half-sweep (colour c) from in into out; with `mean_out`, also
// the volume-weighted mean of out
template <typename T>
__global__ void k_rb_half(LevelView<T> L, const T* __restrict__ in, T* __restrict__ out, int c, double* partial,
                          unsigned* counter, double* mean_out) {
    pdl_entry();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0;
    if (i < L.n) {
        out[i] = L.colour[i] == c ? rb_update(L, in, i) : in[i];
        v = double(L.vol[i]) * double(out[i]);
    }
    if (mean_out) {
        if (publish_partial(v, partial, counter)) {
            double s = fold_partials(partial, gridDim.x);
            if (threadIdx.x == 0) {
                *mean_out = s * L.cvol_inv;
                *counter = 0;
            }
        }
    }
}

// first red-black sweep from zero into out
template <typename T, typename TB>
__global__ void k_rb_pre(LevelView<T> L, const TB* __restrict__ b, const double* level_sum, T* out) {
    pdl_entry();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double mean = (L.singular && level_sum) ? *level_sum * L.cvol_inv : 0.0;
    if (i < L.n) rb_first_cell<T, TB>(L, b, mean, out, i);
}

// one red-black sweep (colour c, then the other) from in into out; with
// `mean_out`, also the volume-weighted mean of out
template <typename T>
__global__ void k_rb_pair(LevelView<T> L, const T* __restrict__ in, T* __restrict__ out, int c, double* partial,
                          unsigned* counter, double* mean_out) {
    pdl_entry();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0;
    if (i < L.n) {
        rb_pair_cell(L, in, out, c, i);
        v = double(L.vol[i]) * double(out[i]);
    }
    if (mean_out) {
        if (publish_partial(v, partial, counter)) {
            double s = fold_partials(partial, gridDim.x);
            if (threadIdx.x == 0) {
                *mean_out = s * L.cvol_inv;
                *counter = 0;
            }
        }
    }
}

template <typename T>
__global__ void k_residual(LevelView<T> L) {
    pdl_entry();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.n) residual_cell(L, i);
}

// b_c = P_tent'(r - wt A s), four threads per coarse cell (grid over 4 nc);
// coarse RHS sum folded into `coarse_sum` when non-null.
template <typename T>
__global__ void k_restrict(LevelView<T> L, T* __restrict__ bc, double* partial, unsigned* counter, double* coarse_sum) {
    pdl_entry();
    // grid-stride over whole warps (the shuffles need every lane of a warp)
    const int quads = (4 * L.nc + 31) & ~31;
    double part = 0;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < quads; g += gridDim.x * blockDim.x) {
        const int J = g >> 2;
        const T v = restrict_quad(L, J, g & 3);
        if ((g & 3) == 0 && J < L.nc) {
            bc[J] = v;
            part += double(v);
        }
    }
    if (coarse_sum) {
        if (publish_partial(part, partial, counter)) {
            double s = fold_partials(partial, gridDim.x);
            if (threadIdx.x == 0) {
                *coarse_sum = s;
                *counter = 0;
            }
        }
    }
}

// Residual and restriction in one launch: b_c = P_tent'(r - wt A Dt^-1 r) with
// r = bp - A x recomputed at every neighbour of a child (four lanes per coarse
// cell, as k_restrict).  Saves the residual phase and the r / s round trip at
// the price of about nnz_row^2 products per fine cell.
template <typename T>
__global__ void k_resrest(LevelView<T> L, T* __restrict__ bc, double* partial, unsigned* counter,
                          double* coarse_sum) {
    pdl_entry();
    const int quads = (4 * L.nc + 31) & ~31;
    double part = 0;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < quads; g += gridDim.x * blockDim.x) {
        const int J = g >> 2, q = g & 3;
        T acc = T(0);
        if (J < L.nc)
            for (int c = L.cptr[J] + q; c < L.cptr[J + 1]; c += 4) {
                const int i = L.child[c];
                const T ri = L.bp[i] - rowdot(L, L.x, i);
                T as = T(0);
                for (int k = L.rp[i]; k < L.rp[i + 1]; ++k) {
                    const int j = L.ci[k];
                    const T rj = j == i ? ri : L.bp[j] - rowdot(L, L.x, j);
                    as += L.val[k] * (L.tinv[j] * rj);
                }
                acc += ri - L.tw * as;
            }
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        acc += __shfl_xor_sync(0xffffffffu, acc, 2);
        if (q == 0 && J < L.nc) {
            bc[J] = acc;
            part += double(acc);
        }
    }
    if (coarse_sum) {
        if (publish_partial(part, partial, counter)) {
            double s = fold_partials(partial, gridDim.x);
            if (threadIdx.x == 0) {
                *coarse_sum = s;
                *counter = 0;
            }
        }
    }
}

template <typename T>
__global__ void k_prolong(LevelView<T> L, const T* __restrict__ xc) {
    pdl_entry();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.n) prolong_cell(L, xc, i);
}

// first post-sweep: y = sweep(x)
template <typename T>
__global__ void k_post1(LevelView<T> L) {
    pdl_entry();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.n) sweep_cell(L, L.x, L.y, i);
}

// second post-sweep x = sweep(y); with `mean_out`, also the volume-weighted mean
template <typename T, typename Epi = MeanOnly>
__global__ void k_post2(LevelView<T> L, double* partial, unsigned* counter, double* mean_out, Epi epi = Epi()) {
    pdl_entry();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0, w = 0;
    if (i < L.n) {
        sweep_cell(L, L.y, L.x, i);
        const double xi = double(L.x[i]);
        v = double(L.vol[i]) * xi;
        if constexpr (Epi::kRz) w = epi.r[i] * xi;
    }
    if (mean_out) fold_mean(v, w, partial, counter, mean_out, L.cvol_inv, epi);
}

// ---------------------------------------------------------------------------------
// coarse tail: levels first..nl-1 in one thread-block cluster (a launch without
// clusters is the one-CTA case).  The CTAs stride the rows of each phase together
// and meet at the hardware cluster barrier between phases (release/acquire at
// cluster scope, which orders their global writes); sums go through distributed
// shared memory in rank order, so every CTA folds the same total.

template <typename T>
__device__ double tail_sum(const T* v, const T* w, int n) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int nb = int(cl.num_blocks());
    double acc = 0;
    for (int i = int(cl.block_rank()) * blockDim.x + threadIdx.x; i < n; i += nb * blockDim.x)
        acc += w ? double(w[i]) * double(v[i]) : double(v[i]);
    const double s = block_sum_all(acc);
    __shared__ double part;
    if (threadIdx.x == 0) part = s;
    cl.sync();
    double total = 0;
    for (int r = 0; r < nb; ++r) total += *cl.map_shared_rank(&part, r);
    cl.sync();  // every CTA has read `part` before the next sum overwrites it
    return total;
}

template <typename T, typename TB>
__device__ void tail_run(const LevelView<T>* __restrict__ levels, int first, int nl, const TB* top_b,
                         const double* __restrict__ G, int gn, double* mean_out);

// `top_b`: RHS of level 0 (type TB), used only when first == 0
template <typename T, typename TB>
__global__ void __launch_bounds__(kTailThreads) k_tail(const LevelView<T>* __restrict__ levels, int first, int nl,
                                                       const TB* top_b, const double* __restrict__ G, int gn,
                                                       double* mean_out) {
    pdl_entry();
    tail_run<T, TB>(levels, first, nl, top_b, G, gn, mean_out);
}

// The tail's levels in the calling cluster (one CTA when launched without clusters).
template <typename T, typename TB>
__device__ void tail_run(const LevelView<T>* __restrict__ levels, int first, int nl, const TB* top_b,
                         const double* __restrict__ G, int gn, double* mean_out) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = int(cl.block_rank()), nb = int(cl.num_blocks());
    const int gt = rank * blockDim.x + threadIdx.x, gs = nb * blockDim.x;
    for (int l = first; l < nl; ++l) {
        LevelView<T> L = levels[l];
        const bool top = (l == 0);  // only the finest level reads the caller's RHS
        double mean = 0;
        if (L.singular) {
            double s = top ? tail_sum(top_b, (const TB*)nullptr, L.n) : tail_sum(L.b, (const T*)nullptr, L.n);
            mean = s * L.cvol_inv;
        }
        if (l == nl - 1) {
            // projected RHS, then the dense (augmented) coarse solve in FP64
            for (int i = gt; i < L.n; i += gs)
                L.bp[i] = top ? proj_b<T, TB>(L, top_b, mean, i) : proj_b<T, T>(L, L.b, mean, i);
            cl.sync();
            // one warp per row, lanes striding the row: coalesced reads of G
            const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
            const int warp = rank * nwarps + (threadIdx.x >> 5);
            for (int i = warp; i < gn; i += nb * nwarps) {
                const double* row = G + size_t(i) * gn;
                double acc = 0;
                for (int k = lane; k < gn; k += 32) acc += row[k] * double(L.bp[k]);
                for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
                if (!lane) L.x[i] = T(acc);
            }
            cl.sync();
            break;
        }
        if (L.rb) {
            for (int i = gt; i < L.n; i += gs) {
                if (top) rb_first_cell<T, TB>(L, top_b, mean, L.y, i);
                else rb_first_cell<T, T>(L, L.b, mean, L.y, i);
            }
            cl.sync();
            for (int i = gt; i < L.n; i += gs) rb_pair_cell(L, L.y, L.x, 0, i);
        } else {
            for (int i = gt; i < L.n; i += gs) {
                if (top) pre2_cell<T, TB>(L, top_b, mean, i);
                else pre2_cell<T, T>(L, L.b, mean, i);
            }
        }
        cl.sync();
        for (int i = gt; i < L.n; i += gs) residual_cell(L, i);
        cl.sync();
        T* bc = levels[l + 1].b;
        // four lanes per coarse cell; the bound is rounded up to whole warps so
        // that every lane of a warp takes part in the shuffles
        const int quads = (4 * L.nc + 31) & ~31;
        for (int g = gt; g < quads; g += gs) {
            const T v = restrict_quad(L, g >> 2, g & 3);
            if ((g & 3) == 0 && (g >> 2) < L.nc) bc[g >> 2] = v;
        }
        cl.sync();
    }
    for (int l = nl - 2; l >= first; --l) {
        LevelView<T> L = levels[l];
        const T* xc = levels[l + 1].x;
        for (int i = gt; i < L.n; i += gs) prolong_cell(L, xc, i);
        cl.sync();
        if (L.rb) {
            for (int i = gt; i < L.n; i += gs) rb_pair_cell(L, L.x, L.y, 1, i);
            cl.sync();
            for (int i = gt; i < L.n; i += gs) rb_pair_cell(L, L.y, L.x, 1, i);
            cl.sync();
            continue;
        }
        for (int i = gt; i < L.n; i += gs) sweep_cell(L, L.x, L.y, i);
        cl.sync();
        for (int i = gt; i < L.n; i += gs) sweep_cell(L, L.y, L.x, i);
        cl.sync();
    }
    if (mean_out && first == 0) {
        LevelView<T> L = levels[0];
        if (L.singular) {
            double s = tail_sum(L.x, L.vol, L.n);
            if (gt == 0) *mean_out = s * L.cvol_inv;
        } else if (gt == 0) {
            *mean_out = 0;
        }
    }
}

}  // namespace tpa
