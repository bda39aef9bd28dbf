// Kernels of the merged batch: many independent pressure solves (uneven tree
// depths) advanced together, one launch per V-cycle phase for every problem.
//
// Batch level j holds, for every problem k with L_k levels, its level
// l = j - (Lmax - L_k) when l >= 0 (levels aligned at the coarse end, so all
// coarsest levels share the last batch level).  Rows are concatenated in
// problem order; CSR columns, owners and child lists use batch-level row
// numbers.  Work is described by items of at most kItemRows rows that never
// straddle two problems (a work list per level), so a CTA's rows belong to one
// problem and per-problem sums fold per-item partials in item order
// (deterministic).  The smoother weight and the transfer weight are folded into
// per-row arrays wd = w D^-1 and td = wt Dt^-1 because they differ between
// problems.
//
// Per problem, the cycle and the CG recurrences are those of the single solve
// (src/solvers/multigrid/cycles.jl:8-77 and Krylov.jl 0.10 `cg!` as called by
// src/solvers/multigrid/elliptic_solver.jl:403-464, ronaldremmerswaal/
// TwoPhaseAMR.jl); a problem that meets its stopping rule is frozen (its
// `active` flag cleared) while the others continue.
#pragma once

#include <climits>
#include <cuda_runtime.h>

#include "fused.cuh"

namespace tpa {

constexpr int kItemRows = 256;
constexpr int kNoExt = INT_MIN;
constexpr int kBatchTailLevels = 4;
constexpr int kBatchTailCells = 2048;  // per problem, for its one-CTA tail

// rows [begin, end) of problem `prob`; delta != kNoExt on a problem's finest
// level, where fine-space index = row + delta
struct BItem {
    int begin, end, prob, delta;
};

// a finest-level item of the CG (fine-space rows [begin, end); level row = row + off)
struct BFItem {
    int begin, end, prob, lvl, off;
};

template <typename T>
struct BLevel {
    int n, nitems;
    const BItem* items;
    const int* rp;
    const int* ci;
    const T* val;
    const T* wd;   // w_k D^-1
    const T* td;   // wt_k Dt^-1
    const T* vol;
    const int* owner;           // row of the next coarser batch level (null on the last)
    const int* cptr;            // children of coarser row J: child[cptr[J] .. cptr[J+1])
    const int* child;
    const double* cvol_inv;     // per problem: 1 / component volume (0: no projection)
    const int* pfirst;          // per problem: first item on this level
    const int* pcount;          // per problem: items on this level (0: absent)
    double* lsum;               // per problem: RHS sum of this level
    T *b, *bp, *x, *y, *r, *s;
};

// per-problem CG scalars (the single solve's CgState)
struct BState {
    double gamma, pAp, alpha, beta, pnorm2, strong_max, target, rsum, rnorm;
    int flags;  // 1 user exit, 2 zero curvature, 4 machine stop, 8 zero initial residual
    int iter, itmax;
};

// per-problem tail (the last kBatchTailLevels or fewer batch levels in one CTA)
struct BTail {
    int begin[kBatchTailLevels], end[kBatchTailLevels];
    const double* G;  // dense inverse of the augmented coarsest matrix (top-left gn x gn)
    int gn;
};

// Publish this CTA's partial (item `blockIdx.x`) and return true in the CTA
// that completes problem-range [first, first + count); `total` (thread 0) then
// holds the fixed-order sum of the range.
__device__ __forceinline__ bool fold_problem(double v, double* partial, unsigned* counter, int first, int count,
                                             double& total) {
    __shared__ bool last;
    v = block_sum_all(v);
    if (threadIdx.x == 0) {
        partial[blockIdx.x] = v;
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        last = (t == unsigned(count) - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    total = fold_partials(partial + first, count);
    if (threadIdx.x == 0) *counter = 0;
    return true;
}

__device__ __forceinline__ bool fold_problem_max(double v, double* partial, unsigned* counter, int first,
                                                 int count, double& total) {
    __shared__ bool last;
    __shared__ double sh[32];
    __shared__ int nan_seen;
    // block max, NaN propagating
    bool nan = v != v;
    double m = nan ? 0.0 : v;
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) nan_seen = 0;
    __syncthreads();
    if (nan) nan_seen = 1;
    if (!lane) sh[wid] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double bm = 0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) bm = fmax(bm, sh[w]);
        partial[blockIdx.x] = nan_seen ? NAN : bm;
        __threadfence();
        unsigned t = atomicAdd(counter, 1u);
        last = (t == unsigned(count) - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    total = fold_partials_max(partial + first, count);
    if (threadIdx.x == 0) *counter = 0;
    return true;
}

template <typename T>
__device__ __forceinline__ T brow(const BLevel<T>& L, const T* v, int i) {
    T acc = T(0);
    for (int k = L.rp[i]; k < L.rp[i + 1]; ++k) acc += L.val[k] * v[L.ci[k]];
    return acc;
}

// ---- V-cycle phases (multi-CTA, one item per CTA) --------------------------------

// both pre-sweeps from x = 0 with the level's RHS projection; on a problem's
// finest level the RHS is the fine-space residual `ext` (FP64) and its sum `ext_sum`
template <typename T>
__global__ void bk_pre2(BLevel<T> L, const double* __restrict__ ext, const BState* __restrict__ st,
                        const int* __restrict__ active) {
    pdl_entry();
    const BItem it = L.items[blockIdx.x];
    if (!active[it.prob]) return;
    const int i = it.begin + int(threadIdx.x);
    if (i >= it.end) return;
    const bool top = it.delta != kNoExt;
    const double sum = top ? st[it.prob].rsum : L.lsum[it.prob];
    const double mean = sum * L.cvol_inv[it.prob];
    auto pb = [&](int q) -> T {
        const double v = top ? ext[q + it.delta] : double(L.b[q]);
        return T(v - double(L.vol[q]) * mean);
    };
    const T bi = pb(i);
    T acc = T(0);
    for (int k = L.rp[i]; k < L.rp[i + 1]; ++k) {
        const int j = L.ci[k];
        const T bj = j == i ? bi : pb(j);
        acc += L.val[k] * (L.wd[j] * bj);
    }
    const T x1 = L.wd[i] * bi;
    L.x[i] = x1 + L.wd[i] * (bi - acc);
    L.bp[i] = bi;
}

template <typename T>
__global__ void bk_residual(BLevel<T> L, const int* __restrict__ active) {
    pdl_entry();
    const BItem it = L.items[blockIdx.x];
    if (!active[it.prob]) return;
    const int i = it.begin + int(threadIdx.x);
    if (i >= it.end) return;
    const T ri = L.bp[i] - brow(L, L.x, i);
    L.r[i] = ri;
    L.s[i] = L.td[i] * ri;
}

// Restriction sum of coarse row J by four lanes (lane q takes children q, q + 4,
// ...), combined in the fixed order (c0 + c1) + (c2 + c3); whole warps call it.
template <typename T>
__device__ __forceinline__ T brestrict_quad(const BLevel<T>& F, int J, bool valid, int q) {
    T v = T(0);
    if (valid)
        for (int k = F.cptr[J] + q; k < F.cptr[J + 1]; k += 4) {
            const int i = F.child[k];
            v += F.r[i] - brow(F, F.s, i);
        }
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    return v;
}

// b_c = P_tent'(r - A s) over the coarse rows of C, one thread per coarse row
// (the merged levels are large: measured faster than four lanes per row);
// per-problem coarse RHS sums
template <typename T>
__global__ void bk_restrict(BLevel<T> F, BLevel<T> C, double* partial, unsigned* counters,
                            const int* __restrict__ active) {
    pdl_entry();
    const BItem it = C.items[blockIdx.x];
    if (!active[it.prob]) return;
    const int J = it.begin + int(threadIdx.x);
    T v = T(0);
    if (J < it.end) {
        for (int k = F.cptr[J]; k < F.cptr[J + 1]; ++k) {
            const int i = F.child[k];
            v += F.r[i] - brow(F, F.s, i);
        }
        C.b[J] = v;
    }
    double total;
    if (fold_problem(double(v), partial, counters + it.prob, C.pfirst[it.prob], C.pcount[it.prob], total) &&
        threadIdx.x == 0)
        C.lsum[it.prob] = total;
}

template <typename T>
__global__ void bk_prolong(BLevel<T> L, const T* __restrict__ xc, const int* __restrict__ active) {
    pdl_entry();
    const BItem it = L.items[blockIdx.x];
    if (!active[it.prob]) return;
    const int i = it.begin + int(threadIdx.x);
    if (i >= it.end) return;
    T ae = T(0);
    for (int k = L.rp[i]; k < L.rp[i + 1]; ++k) ae += L.val[k] * xc[L.owner[L.ci[k]]];
    L.x[i] += xc[L.owner[i]] - L.td[i] * ae;
}

template <typename T>
__global__ void bk_post1(BLevel<T> L, const int* __restrict__ active) {
    pdl_entry();
    const BItem it = L.items[blockIdx.x];
    if (!active[it.prob]) return;
    const int i = it.begin + int(threadIdx.x);
    if (i >= it.end) return;
    L.y[i] = L.x[i] + L.wd[i] * (L.bp[i] - brow(L, L.x, i));
}

// second post-sweep; on a problem's finest level also its volume-weighted mean
template <typename T>
__global__ void bk_post2(BLevel<T> L, double* partial, unsigned* counters, double* __restrict__ mean_out,
                         const int* __restrict__ active) {
    pdl_entry();
    const BItem it = L.items[blockIdx.x];
    if (!active[it.prob]) return;
    const int i = it.begin + int(threadIdx.x);
    double v = 0;
    if (i < it.end) {
        const T xi = L.y[i] + L.wd[i] * (L.bp[i] - brow(L, L.y, i));
        L.x[i] = xi;
        v = double(L.vol[i]) * double(xi);
    }
    if (it.delta == kNoExt) return;
    double total;
    if (fold_problem(v, partial, counters + it.prob, L.pfirst[it.prob], L.pcount[it.prob], total) &&
        threadIdx.x == 0)
        mean_out[it.prob] = total * L.cvol_inv[it.prob];
}

// ---- per-problem tail: one CTA runs a problem's last batch levels ----------------

template <typename T>
__device__ double btail_sum(const T* v, const T* w, int b, int e) {
    double acc = 0;
    for (int i = b + int(threadIdx.x); i < e; i += blockDim.x) acc += w ? double(w[i]) * double(v[i]) : double(v[i]);
    __syncthreads();
    double s = block_sum_all(acc);
    __shared__ double total;
    if (threadIdx.x == 0) total = s;
    __syncthreads();
    return total;
}

// levels: the batch levels first .. first + nt - 1 (device array of views)
template <typename T>
__global__ void __launch_bounds__(kTailThreads) bk_tail(const BLevel<T>* __restrict__ levels, int first, int nt,
                                                        const BTail* __restrict__ tails,
                                                        const int* __restrict__ active) {
    pdl_entry();
    const int k = blockIdx.x;
    if (!active[k]) return;
    const BTail tl = tails[k];
    if (tl.gn == 0) return;  // the problem has no levels here (cannot happen: all share the last level)
    for (int t = 0; t < nt; ++t) {
        const BLevel<T> L = levels[first + t];
        const int b0 = tl.begin[t], e0 = tl.end[t];
        double mean = 0;
        const double cv = L.cvol_inv[k];
        if (cv != 0) mean = btail_sum(L.b, (const T*)nullptr, b0, e0) * cv;
        if (t == nt - 1) {
            for (int i = b0 + int(threadIdx.x); i < e0; i += blockDim.x)
                L.bp[i] = T(double(L.b[i]) - double(L.vol[i]) * mean);
            __syncthreads();
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
            for (int i = warp; i < tl.gn; i += nwarps) {
                const double* row = tl.G + size_t(i) * tl.gn;
                double acc = 0;
                for (int c = lane; c < tl.gn; c += 32) acc += row[c] * double(L.bp[b0 + c]);
                for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
                if (!lane) L.x[b0 + i] = T(acc);
            }
            __syncthreads();
            break;
        }
        for (int i = b0 + int(threadIdx.x); i < e0; i += blockDim.x) {
            auto pb = [&](int q) -> T { return T(double(L.b[q]) - double(L.vol[q]) * mean); };
            const T bi = pb(i);
            T acc = T(0);
            for (int c = L.rp[i]; c < L.rp[i + 1]; ++c) {
                const int j = L.ci[c];
                acc += L.val[c] * (L.wd[j] * (j == i ? bi : pb(j)));
            }
            L.x[i] = L.wd[i] * bi + L.wd[i] * (bi - acc);
            L.bp[i] = bi;
        }
        __syncthreads();
        for (int i = b0 + int(threadIdx.x); i < e0; i += blockDim.x) {
            const T ri = L.bp[i] - brow(L, L.x, i);
            L.r[i] = ri;
            L.s[i] = L.td[i] * ri;
        }
        __syncthreads();
        const BLevel<T> C = levels[first + t + 1];
        {
            // four lanes per coarse row, over whole warps
            const int cb = tl.begin[t + 1], nc = tl.end[t + 1] - cb;
            const int quads = (4 * nc + 31) & ~31;
            for (int g = int(threadIdx.x); g < quads; g += blockDim.x) {
                const int J = cb + (g >> 2);
                const T v = brestrict_quad(L, J, (g >> 2) < nc, g & 3);
                if ((g & 3) == 0 && (g >> 2) < nc) C.b[J] = v;
            }
        }
        __syncthreads();
    }
    for (int t = nt - 2; t >= 0; --t) {
        const BLevel<T> L = levels[first + t];
        const T* xc = levels[first + t + 1].x;
        const int b0 = tl.begin[t], e0 = tl.end[t];
        for (int i = b0 + int(threadIdx.x); i < e0; i += blockDim.x) {
            T ae = T(0);
            for (int c = L.rp[i]; c < L.rp[i + 1]; ++c) ae += L.val[c] * xc[L.owner[L.ci[c]]];
            L.x[i] += xc[L.owner[i]] - L.td[i] * ae;
        }
        __syncthreads();
        for (int i = b0 + int(threadIdx.x); i < e0; i += blockDim.x)
            L.y[i] = L.x[i] + L.wd[i] * (L.bp[i] - brow(L, L.x, i));
        __syncthreads();
        for (int i = b0 + int(threadIdx.x); i < e0; i += blockDim.x)
            L.x[i] = L.y[i] + L.wd[i] * (L.bp[i] - brow(L, L.y, i));
        __syncthreads();
    }
}

}  // namespace tpa
