// The CMDGFM two-block solve on the device (cmdgfm.cuh).
//
// ronaldremmerswaal/TwoPhaseAMR.jl solves the assembled system in
// `_project_cmdgfm_assembled!` (src/two_phase/projection/cmdgfm_projection.jl:
// 2201-2291): residual replacement around Krylov.jl 0.10 `bicgstab!` runs on
// the diagonally scaled system D_r M D_c (`_cmdgfm_krylov_scaling!`, :215-235)
// with the block preconditioner of :411-441 -- one V-cycle of the pressure
// hierarchy on the reduced pressure block (:374-405) and the incomplete LU of
// J - C D^-1 B on the jump block.  Here every vector lives in HBM, the
// V-cycle is the context's device cycle, the factor's triangular solves run
// level by level in one CTA with the vector in shared memory, and every
// reduction is a fixed-order fold of per-block partials (one block folds), so
// a solve repeats bit for bit.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "cmdgfm.cuh"

namespace tpa {
namespace {

constexpr int kT = 256;
constexpr int kG = 1184;  // 8 CTAs of 256 threads on each of 148 SMs
constexpr int kIluThreads = 1024;

inline int grid_of(int64_t n) {
    return int(std::max<int64_t>(1, std::min<int64_t>((n + kT - 1) / kT, kG)));
}

#define CM_LOOP(i, n) \
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < (n); i += int64_t(gridDim.x) * blockDim.x)

// state slots
enum : int {
    kRho = 0, kNextRho, kAlpha, kOmega, kBeta, kRnorm, kEps, kIter, kItmax, kFlags,
    kPressureDefect, kJumpDefect, kAnchorDefect, kRhsNorm2, kNonfinite, kChanged, kNorm2, kStateSize
};
enum : int { kSolved = 1, kTired = 2, kBreakdown = 4, kZeroRhs = 8, kZeroRho = 16 };

__device__ __forceinline__ double block_max_all(double v) {
    __shared__ double sh[32];
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (!lane) sh[wid] = v;
    __syncthreads();
    v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    if (wid == 0)
        for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// a NaN anywhere makes the maximum NaN
__device__ __forceinline__ double nan_max(double a, double b) { return (a != a || b != b) ? NAN : fmax(a, b); }

// ---------------------------------------------------------------- preconditioner

// full[cell_i] = src_i / rows_i (the reduced right-hand side scattered); with
// one component (anchor >= 0) the last block also writes full[anchor] = -(the
// sum of the values), folded from per-block partials in block order
__global__ void k_cm_scatter(int64_t np, const double* __restrict__ src, const double* __restrict__ rows,
                             const int32_t* __restrict__ cell, double* __restrict__ full, int anchor,
                             double* partial, unsigned* counter) {
    double v = 0;
    CM_LOOP(i, np) {
        const double q = src[i] / rows[i];
        full[cell[i]] = q;
        v += q;
    }
    if (anchor < 0) return;
    if (publish_partial(v, partial, counter)) {
        const double t = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            full[anchor] = 0.0 - t;
            *counter = 0;
        }
    }
}

// one block per anchor: full[anchor] = -(sum of its component's values)
__global__ void k_cm_anchor(const int32_t* __restrict__ gptr, const int32_t* __restrict__ gidx,
                            const int32_t* __restrict__ ganchor, const double* __restrict__ src,
                            const double* __restrict__ rows, double* __restrict__ full) {
    const int g = blockIdx.x;
    double v = 0;
    for (int k = gptr[g] + threadIdx.x; k < gptr[g + 1]; k += blockDim.x) {
        const int i = gidx[k];
        v += src[i] / rows[i];
    }
    v = block_sum_all(v);
    if (threadIdx.x == 0) full[ganchor[g]] = 0.0 - v;
}

// zp_i = z[cell_i] - z[anchor_i]; dst_i = zp_i / cols_i
__global__ void k_cm_gather(int64_t np, const double* __restrict__ z, const int32_t* __restrict__ cell,
                            const int32_t* __restrict__ anchor, const double* __restrict__ cols,
                            double* __restrict__ zp, double* __restrict__ dst) {
    CM_LOOP(i, np) {
        const double v = z[cell[i]] - z[anchor[i]];
        zp[i] = v;
        dst[i] = v / cols[i];
    }
}

// One factor of the jump block laid out for its triangular solve: position i
// holds row rows[i], its entries (col, val)[ptr[i] .. ptr[i+1]) in column
// order and, for U, the reciprocal of its pivot inv[i].  `seq`: the positions
// are the rows in solve order (increasing for L, decreasing for U) and one
// thread walks them; otherwise the rows of level v are positions lev[v] ..
// lev[v+1], independent of each other, and the CTA takes each level between
// barriers.  A schedule whose levels hold few rows each -- the chains along
// the interface -- runs faster on one thread than with a barrier per level.

// copy a factor's arrays into shared memory at `at`; returns the view of the
// copy and advances `at` (8-byte aligned: doubles first)
template <bool Upper>
__device__ TriView stage(const TriView& g, int nx, char*& at) {
    TriView t = g;
    double* val = reinterpret_cast<double*>(at);
    double* inv = val + g.nnz;
    int32_t* lev = reinterpret_cast<int32_t*>(inv + (Upper ? nx : 0));
    int32_t* rows = lev + g.nlev + 1;
    int32_t* ptr = rows + nx;
    int32_t* col = ptr + nx + 1;
    for (int e = threadIdx.x; e < g.nnz; e += blockDim.x) {
        val[e] = g.val[e];
        col[e] = g.col[e];
    }
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        rows[i] = g.rows[i];
        if (Upper) inv[i] = g.inv[i];
    }
    for (int i = threadIdx.x; i <= nx; i += blockDim.x) ptr[i] = g.ptr[i];
    for (int i = threadIdx.x; i <= g.nlev; i += blockDim.x) lev[i] = g.lev[i];
    t.val = val;
    t.inv = inv;
    t.lev = lev;
    t.rows = rows;
    t.ptr = ptr;
    t.col = col;
    at = reinterpret_cast<char*>(col + g.nnz);
    at += (8 - (reinterpret_cast<size_t>(at) & 7)) & 7;
    return t;
}

// The rows in solve order on one thread.  The next row's index, extent and
// first kPre entries are loaded into registers while the current row is
// summed, and the value just computed stays in a register for the next row,
// which in a chain along the interface usually needs it: the critical path
// per row is then one multiply-add and the reads of older values.
template <bool Upper>
__device__ __forceinline__ void walk_rows(double* __restrict__ y, const double* __restrict__ val,
                                          const double* __restrict__ inv, const int32_t* __restrict__ rows,
                                          const int32_t* __restrict__ ptr, const int32_t* __restrict__ col, int nx) {
    constexpr int kPre = 4;
    if (nx <= 0) return;
    int k = rows[0], e0 = ptr[0], e1 = ptr[1];
    int c[kPre];
    double v[kPre];
    for (int q = 0; q < kPre; ++q) {
        c[q] = e0 + q < e1 ? col[e0 + q] : 0;
        v[q] = e0 + q < e1 ? val[e0 + q] : 0.0;
    }
    double w = Upper ? inv[0] : 1.0;
    int klast = -1;
    double ylast = 0.0;
    for (int i = 0; i < nx; ++i) {
        const bool more = i + 1 < nx;
        const int nk = more ? rows[i + 1] : 0;
        const int ne1 = more ? ptr[i + 2] : e1;
        const double nw = (Upper && more) ? inv[i + 1] : 1.0;
        int nc[kPre];
        double nv[kPre];
        for (int q = 0; q < kPre; ++q) {
            nc[q] = e1 + q < ne1 ? col[e1 + q] : 0;
            nv[q] = e1 + q < ne1 ? val[e1 + q] : 0.0;
        }
        double acc = y[k];
        for (int q = 0; q < kPre; ++q)
            if (e0 + q < e1) {
                double yc;
                if (c[q] == klast) yc = ylast;
                else yc = y[c[q]];
                acc -= v[q] * yc;
            }
        for (int e = e0 + kPre; e < e1; ++e) acc -= val[e] * (col[e] == klast ? ylast : y[col[e]]);
        const double yk = Upper ? acc * w : acc;
        y[k] = yk;
        klast = k;
        ylast = yk;
        k = nk;
        e0 = e1;
        e1 = ne1;
        w = nw;
        for (int q = 0; q < kPre; ++q) {
            c[q] = nc[q];
            v[q] = nv[q];
        }
    }
}

template <bool Upper>
__device__ void tri_solve(const TriView& t, double* __restrict__ y, int nx) {
    auto row = [&](int i) {
        const int k = t.rows[i];
        double acc = y[k];
        for (int e = t.ptr[i]; e < t.ptr[i + 1]; ++e) acc -= t.val[e] * y[t.col[e]];
        y[k] = Upper ? acc * t.inv[i] : acc;
    };
    if (t.seq) {
        if (threadIdx.x == 0) walk_rows<Upper>(y, t.val, t.inv, t.rows, t.ptr, t.col, nx);
    } else {
        for (int v = 0; v < t.nlev; ++v) {
            for (int i = t.lev[v] + int(threadIdx.x); i < t.lev[v + 1]; i += blockDim.x) row(i);
            __syncthreads();
        }
    }
    __syncthreads();
}

// The jump block of the block preconditioner in one CTA: jr = src_xi / D_r -
// C zp, y = (L U)^-1 jr, dst_xi = y / D_c.  The vector lives in shared
// memory, and the factors too when `staged`.
__global__ void __launch_bounds__(kIluThreads)
    k_cm_jump_solve(int nx, int64_t np, const double* __restrict__ src, const double* __restrict__ rows,
                    const int64_t* __restrict__ cptr, const int32_t* __restrict__ ccol,
                    const double* __restrict__ cval, const double* __restrict__ zp, TriView L, TriView U,
                    int staged, const double* __restrict__ cols, double* __restrict__ dst) {
    extern __shared__ double sm[];
    double* y = sm;
    for (int f = threadIdx.x; f < nx; f += blockDim.x) {
        double acc = 0;
        for (int64_t e = cptr[f]; e < cptr[f + 1]; ++e) acc += cval[e] * zp[ccol[e]];
        y[f] = src[np + f] / rows[np + f] - acc;
    }
    if (staged) {
        char* at = reinterpret_cast<char*>(y + nx);
        L = stage<false>(L, nx, at);
        U = stage<true>(U, nx, at);
    }
    __syncthreads();
    if (staged && L.seq && U.seq) {
        // both factors walked on one thread, every array in shared memory
        if (threadIdx.x == 0) {
            const double* lval = reinterpret_cast<const double*>(y + nx);
            const int32_t* llev = reinterpret_cast<const int32_t*>(lval + L.nnz);
            const int32_t* lrows = llev + L.nlev + 1;
            const int32_t* lptr = lrows + nx;
            const int32_t* lcol = lptr + nx + 1;
            walk_rows<false>(y, lval, nullptr, lrows, lptr, lcol, nx);
            const char* at = reinterpret_cast<const char*>(lcol + L.nnz);
            at += (8 - (reinterpret_cast<size_t>(at) & 7)) & 7;
            const double* uval = reinterpret_cast<const double*>(at);
            const double* uinv = uval + U.nnz;
            const int32_t* ulev = reinterpret_cast<const int32_t*>(uinv + nx);
            const int32_t* urows = ulev + U.nlev + 1;
            const int32_t* uptr = urows + nx;
            const int32_t* ucol = uptr + nx + 1;
            walk_rows<true>(y, uval, uinv, urows, uptr, ucol, nx);
        }
        __syncthreads();
    } else {
        tri_solve<false>(L, y, nx);
        tri_solve<true>(U, y, nx);
    }
    for (int f = threadIdx.x; f < nx; f += blockDim.x) dst[np + f] = y[f] / cols[np + f];
}

// The jump block through the factors' inverses (triangular_inverses): jr =
// src_xi / D_r - C zp, y = L^-1 jr, x = U^-1 y, dst_xi = x / D_c, each a
// row-parallel product; one CTA, jr and y in shared memory.
__global__ void __launch_bounds__(kIluThreads)
    k_cm_jump_inverse(int nx, int64_t np, const double* __restrict__ src, const double* __restrict__ rows,
                      const int64_t* __restrict__ cptr, const int32_t* __restrict__ ccol,
                      const double* __restrict__ cval, const double* __restrict__ zp,
                      const int64_t* __restrict__ lptr, const int32_t* __restrict__ lcol,
                      const double* __restrict__ lval, const int64_t* __restrict__ uptr,
                      const int32_t* __restrict__ ucol, const double* __restrict__ uval,
                      const double* __restrict__ cols, double* __restrict__ dst) {
    extern __shared__ double sm[];
    double* a = sm;
    double* b = sm + nx;
    for (int f = threadIdx.x; f < nx; f += blockDim.x) {
        double acc = 0;
        for (int64_t e = cptr[f]; e < cptr[f + 1]; ++e) acc += cval[e] * zp[ccol[e]];
        a[f] = src[np + f] / rows[np + f] - acc;
    }
    __syncthreads();
    for (int f = threadIdx.x; f < nx; f += blockDim.x) {
        double acc = 0;
        for (int64_t e = lptr[f]; e < lptr[f + 1]; ++e) acc += lval[e] * a[lcol[e]];
        b[f] = acc;
    }
    __syncthreads();
    for (int f = threadIdx.x; f < nx; f += blockDim.x) {
        double acc = 0;
        for (int64_t e = uptr[f]; e < uptr[f + 1]; ++e) acc += uval[e] * b[ucol[e]];
        dst[np + f] = acc / cols[np + f];
    }
}

// ---------------------------------------------------------------- products

// y = D_r M (D_c x) (scaled) or y = M x (rows, cols null)
__global__ void k_cm_spmv(int64_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ col,
                          const double* __restrict__ val, const double* __restrict__ rows,
                          const double* __restrict__ cols, const double* __restrict__ x, double* __restrict__ y) {
    CM_LOOP(i, n) {
        double acc = 0;
        if (cols)
            for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e) acc += val[e] * (cols[col[e]] * x[col[e]]);
        else
            for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e) acc += val[e] * x[col[e]];
        y[i] = rows ? rows[i] * acc : acc;
    }
}

// corr = rhs - M sol
__global__ void k_cm_residual(int64_t n, const int64_t* __restrict__ ptr, const int32_t* __restrict__ col,
                              const double* __restrict__ val, const double* __restrict__ rhs,
                              const double* __restrict__ sol, double* __restrict__ corr) {
    CM_LOOP(i, n) {
        double acc = 0;
        for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e) acc += val[e] * sol[col[e]];
        corr[i] = rhs[i] - acc;
    }
}

// block partials of a'b and c'd (c, d may be null)
__global__ void k_cm_dot2(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                          const double* __restrict__ c, const double* __restrict__ d, double* __restrict__ p1,
                          double* __restrict__ p2) {
    double v = 0, w = 0;
    CM_LOOP(i, n) {
        v += a[i] * b[i];
        if (c) w += c[i] * d[i];
    }
    v = block_sum_all(v);
    if (c) w = block_sum_all(w);
    if (threadIdx.x == 0) {
        p1[blockIdx.x] = v;
        if (c) p2[blockIdx.x] = w;
    }
}

// ---------------------------------------------------------------- BiCGSTAB

// x = 0, r = p = b, v = 0, with the partials of r'r (= c'r: the shadow
// residual c is b itself)
__global__ void k_cm_init(int64_t n, const double* __restrict__ b, double* __restrict__ x, double* __restrict__ r,
                          double* __restrict__ p, double* __restrict__ v, double* __restrict__ p1) {
    double w = 0;
    CM_LOOP(i, n) {
        const double bi = b[i];
        x[i] = 0.0;
        r[i] = bi;
        p[i] = bi;
        v[i] = 0.0;
        w += bi * bi;
    }
    w = block_sum_all(w);
    if (threadIdx.x == 0) p1[blockIdx.x] = w;
}

// rNorm, eps = atol + rtol rNorm, rho_1 = c'r (= rNorm^2: c = r = b)
__global__ void k_cm_init_fold(const double* p1, int count, double rtol, int itmax, double* st) {
    const double rr = fold_partials(p1, count);
    if (threadIdx.x == 0) {
        const double rnorm = sqrt(rr);
        st[kRnorm] = rnorm;
        st[kEps] = 0.0 + rtol * rnorm;
        st[kNextRho] = rr;
        st[kIter] = 0;
        st[kItmax] = itmax;
        int flags = 0;
        if (rnorm == 0.0) flags |= kZeroRhs;
        else if (rr == 0.0) flags |= kZeroRho;
        if (rnorm <= st[kEps]) flags |= kSolved;
        if (itmax <= 0) flags |= kTired;
        st[kFlags] = flags;
    }
}

// rho = next_rho; alpha = rho / c'v
__global__ void k_cm_alpha(const double* p1, int count, double* st) {
    const double cv = fold_partials(p1, count);
    if (threadIdx.x == 0) {
        st[kRho] = st[kNextRho];
        st[kAlpha] = st[kRho] / cv;
    }
}

// s = r - alpha v; x = x + alpha y
__global__ void k_cm_update1(int64_t n, const double* __restrict__ r, const double* __restrict__ v,
                             const double* __restrict__ y, double* __restrict__ s, double* __restrict__ x,
                             const double* __restrict__ st) {
    const double a = st[kAlpha];
    CM_LOOP(i, n) {
        s[i] = r[i] - a * v[i];
        x[i] = x[i] + a * y[i];
    }
}

// omega = t's / t't
__global__ void k_cm_omega(const double* p1, const double* p2, int count, double* st) {
    const double ts = fold_partials(p1, count);
    const double tt = fold_partials(p2, count);
    if (threadIdx.x == 0) st[kOmega] = ts / tt;
}

// x = x + omega z; r = s - omega t; partials of c'r and r'r
__global__ void k_cm_update2(int64_t n, const double* __restrict__ s, const double* __restrict__ t,
                             const double* __restrict__ z, const double* __restrict__ c, double* __restrict__ x,
                             double* __restrict__ r, const double* __restrict__ st, double* __restrict__ p1,
                             double* __restrict__ p2) {
    const double w = st[kOmega];
    double cr = 0, rr = 0;
    CM_LOOP(i, n) {
        x[i] = x[i] + w * z[i];
        const double ri = s[i] - w * t[i];
        r[i] = ri;
        cr += c[i] * ri;
        rr += ri * ri;
    }
    cr = block_sum_all(cr);
    rr = block_sum_all(rr);
    if (threadIdx.x == 0) {
        p1[blockIdx.x] = cr;
        p2[blockIdx.x] = rr;
    }
}

// next_rho, beta, rNorm and the stopping rules of the iteration
__global__ void k_cm_rho(const double* p1, const double* p2, int count, double* st,
                         cudaGraphConditionalHandle handle, int set_cond) {
    const double cr = fold_partials(p1, count);
    const double rr = fold_partials(p2, count);
    if (threadIdx.x == 0) {
        st[kNextRho] = cr;
        st[kBeta] = (cr / st[kRho]) * (st[kAlpha] / st[kOmega]);
        const double rnorm = sqrt(rr);
        st[kRnorm] = rnorm;
        const double iter = st[kIter] + 1;
        st[kIter] = iter;
        int flags = 0;
        if (rnorm <= st[kEps] || rnorm + 1.0 <= 1.0) flags |= kSolved;
        if (iter >= st[kItmax]) flags |= kTired;
        const double a = st[kAlpha];
        if (a == 0.0 || a != a) flags |= kBreakdown;
        st[kFlags] = flags;
        if (set_cond) cudaGraphSetConditional(handle, (flags & (kSolved | kTired | kBreakdown)) ? 0u : 1u);
    }
}

// p = r + beta (p - omega v)
__global__ void k_cm_pupdate(int64_t n, const double* __restrict__ r, const double* __restrict__ v,
                             double* __restrict__ p, const double* __restrict__ st) {
    const double b = st[kBeta], w = st[kOmega];
    CM_LOOP(i, n) p[i] = r[i] + b * (p[i] - w * v[i]);
}

// ---------------------------------------------------------------- residual replacement

// block partials: max weighted |corr| over pressure rows (p1), over jump rows
// (p2), and sum (rows corr)^2 (p3)
__global__ void k_cm_defects(int64_t n, int64_t np, const double* __restrict__ corr,
                             const double* __restrict__ weight, const double* __restrict__ rows, double* __restrict__ p1,
                             double* __restrict__ p2, double* __restrict__ p3) {
    double mp = 0, mj = 0, s2 = 0;
    CM_LOOP(i, n) {
        const double d = weight[i] * fabs(corr[i]);
        if (i < np) mp = nan_max(mp, d);
        else mj = nan_max(mj, d);
        const double q = rows[i] * corr[i];
        s2 += q * q;
    }
    bool nanp = mp != mp, nanj = mj != mj;
    mp = block_max_all(nanp ? 0.0 : mp);
    mj = block_max_all(nanj ? 0.0 : mj);
    s2 = block_sum_all(s2);
    __shared__ int any[2];
    if (threadIdx.x == 0) any[0] = any[1] = 0;
    __syncthreads();
    if (nanp) any[0] = 1;
    if (nanj) any[1] = 1;
    __syncthreads();
    if (threadIdx.x == 0) {
        p1[blockIdx.x] = any[0] ? NAN : mp;
        p2[blockIdx.x] = any[1] ? NAN : mj;
        p3[blockIdx.x] = s2;
    }
}

// the omitted anchor rows at the current solution: block maxima of
// weight_a |rhs_a - (E sol)_a|
__global__ void k_cm_anchor_defect(int64_t na, const int64_t* __restrict__ ptr, const int32_t* __restrict__ col,
                                   const double* __restrict__ val, const double* __restrict__ rhs,
                                   const double* __restrict__ w, const double* __restrict__ sol,
                                   double* __restrict__ p4) {
    double m = 0;
    bool nan = false;
    CM_LOOP(a, na) {
        double acc = 0;
        for (int64_t e = ptr[a]; e < ptr[a + 1]; ++e) acc += val[e] * sol[col[e]];
        const double d = w[a] * fabs(rhs[a] - acc);
        if (d != d) nan = true;
        else m = fmax(m, d);
    }
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    if (nan) any = 1;
    m = block_max_all(m);
    if (threadIdx.x == 0) p4[blockIdx.x] = any ? NAN : m;
}

__device__ double fold_max(const double* p, int count) {
    double m = 0;
    bool nan = false;
    for (int k = threadIdx.x; k < count; k += blockDim.x) {
        const double v = ((volatile const double*)p)[k];
        if (v != v) nan = true;
        else m = fmax(m, v);
    }
    __shared__ int any;
    __syncthreads();  // a previous call's readers of `any` are done
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    if (nan) any = 1;
    m = block_max_all(m);
    __syncthreads();
    return any ? NAN : m;
}

__global__ void k_cm_defects_fold(const double* p1, const double* p2, const double* p3, int count,
                                  const double* p4, int count4, double* st) {
    const double mp = fold_max(p1, count);
    const double mj = fold_max(p2, count);
    const double s2 = fold_partials(p3, count);
    const double ma = count4 > 0 ? fold_max(p4, count4) : 0.0;
    if (threadIdx.x == 0) {
        st[kPressureDefect] = mp;
        st[kJumpDefect] = mj;
        st[kRhsNorm2] = s2;
        st[kAnchorDefect] = ma;
    }
}

// b = rows corr, divided by `norm` when normalize
__global__ void k_cm_scaled_rhs(int64_t n, const double* __restrict__ rows, const double* __restrict__ corr,
                                double* __restrict__ b, int normalize, double norm) {
    CM_LOOP(i, n) {
        const double v = rows[i] * corr[i];
        b[i] = normalize ? v / norm : v;
    }
}

// block partials: non-finite entries of x (p1)
__global__ void k_cm_nonfinite(int64_t n, const double* __restrict__ x, double* __restrict__ p1) {
    double c = 0;
    CM_LOOP(i, n) if (!isfinite(x[i])) c += 1.0;
    c = block_sum_all(c);
    if (threadIdx.x == 0) p1[blockIdx.x] = c;
}

// sol = sol + cols (scale x), block partials of the changed entries (p1)
__global__ void k_cm_apply(int64_t n, double* __restrict__ sol, const double* __restrict__ cols, double scale,
                           const double* __restrict__ x, double* __restrict__ p1) {
    double c = 0;
    CM_LOOP(i, n) {
        const double prev = sol[i];
        const double upd = prev + cols[i] * (scale * x[i]);
        sol[i] = upd;
        if (upd != prev) c += 1.0;
    }
    c = block_sum_all(c);
    if (threadIdx.x == 0) p1[blockIdx.x] = c;
}

__global__ void k_cm_sum_fold(const double* p1, int count, double* out) {
    const double v = fold_partials(p1, count);
    if (threadIdx.x == 0) *out = v;
}

}  // namespace

// ---------------------------------------------------------------- host driver

void CmdgfmDevice::spmv(const double* x, double* y, int mode, cudaStream_t s) {
    // mode 1: the scaled system D_r M D_c; 0: M
    k_cm_spmv<<<grid_of(n_), kT, 0, s>>>(n_, mptr_.p, mcol_.p, mval_.p, mode ? rows_.p : nullptr,
                                         mode ? cols_.p : nullptr, x, y);
    ++launches_;
}

// dst = (N^-1 (src / D_r)) / D_c: `_ScaledProjectionPreconditioner` around
// the block preconditioner (cmdgfm_projection.jl:158-179, 374-441)
void CmdgfmDevice::precondition(DeviceSolver& ds, const CmdgfmFactor& f, const double* src, double* dst,
                                int precision, cudaStream_t s) {
    if (np_ > 0) {
        TPA_CUDA(cudaMemsetAsync(full_.p, 0, sizeof(double) * size_t(ncells_), s));
        // one component: the anchor's value folds in the scatter; several: one block each
        k_cm_scatter<<<grid_of(np_), kT, 0, s>>>(np_, src, rows_.p, cell_.p, full_.p, ngroups_ == 1 ? anchor1_ : -1,
                                                 partial_.p + 2 * kG, counter_.p);
        ++launches_;
        if (ngroups_ > 1) {
            k_cm_anchor<<<ngroups_, 1024, 0, s>>>(gptr_.p, gidx_.p, ganchor_.p, src, rows_.p, full_.p);
            ++launches_;
        }
        const int before = ds.kernel_launches();
        ds.vcycle(full_.p, zfull_.p, precision);
        launches_ += ds.kernel_launches() - before;
        k_cm_gather<<<grid_of(np_), kT, 0, s>>>(np_, zfull_.p, cell_.p, anchor_.p, cols_.p, zp_.p, dst);
        ++launches_;
    }
    if (nx_ > 0) jump_apply(src, rows_.p, cols_.p, zp_.p, dst, s);
    (void)f;
}

// One BiCGSTAB iteration (Krylov.jl 0.10 `bicgstab!` with the right
// preconditioner N): y = N^-1 p, v = A y, alpha; s = r - alpha v, x += alpha y;
// z = N^-1 s, t = A z, omega; x += omega z, r = s - omega t; next rho, beta,
// rNorm and the stopping rules (which set the loop condition when `set_cond`);
// p = r + beta (p - omega v).
void CmdgfmDevice::enqueue_iteration(DeviceSolver& ds, const CmdgfmFactor& f, bool preconditioned, int precision,
                                     cudaStream_t s, cudaGraphConditionalHandle handle, int set_cond) {
    const int g = grid_of(n_);
    double* p1 = partial_.p;
    double* p2 = partial_.p + kG;
    double* st = state_.p;
    const double* y = p_.p;
    if (preconditioned) {
        precondition(ds, f, p_.p, y_.p, precision, s);
        y = y_.p;
    }
    spmv(y, v_.p, 1, s);
    k_cm_dot2<<<g, kT, 0, s>>>(n_, c_.p, v_.p, nullptr, nullptr, p1, nullptr);
    k_cm_alpha<<<1, kT, 0, s>>>(p1, g, st);
    k_cm_update1<<<g, kT, 0, s>>>(n_, r_.p, v_.p, y, s_.p, x_.p, st);
    launches_ += 3;
    const double* z = s_.p;
    if (preconditioned) {
        precondition(ds, f, s_.p, z_.p, precision, s);
        z = z_.p;
    }
    spmv(z, t_.p, 1, s);
    k_cm_dot2<<<g, kT, 0, s>>>(n_, t_.p, s_.p, t_.p, t_.p, p1, p2);
    k_cm_omega<<<1, kT, 0, s>>>(p1, p2, g, st);
    k_cm_update2<<<g, kT, 0, s>>>(n_, s_.p, t_.p, z, c_.p, x_.p, r_.p, st, p1, p2);
    k_cm_rho<<<1, kT, 0, s>>>(p1, p2, g, st, handle, set_cond);
    k_cm_pupdate<<<g, kT, 0, s>>>(n_, r_.p, v_.p, p_.p, st);
    launches_ += 5;
}

// The iteration captured as the body of a graph WHILE node, kept while every
// argument it captured is unchanged: the sizes, the jump-block layout, the
// buffers and the pressure hierarchy's graph generation.
cudaGraphExec_t CmdgfmDevice::loop_graph(DeviceSolver& ds, const CmdgfmFactor& f, bool preconditioned, int precision,
                                         cudaStream_t s) {
    std::vector<uintptr_t> key = {
        uintptr_t(n_), uintptr_t(np_), uintptr_t(nx_), uintptr_t(ncells_), uintptr_t(ngroups_),
        uintptr_t(int64_t(anchor1_)), uintptr_t(precision), uintptr_t(inverse_), uintptr_t(jstaged_),
        uintptr_t(jsmem_), uintptr_t(ds.graph_generation()), uintptr_t(s)};
    for (const void* q : {(const void*)mptr_.p, (const void*)mcol_.p, (const void*)mval_.p, (const void*)rows_.p,
                          (const void*)cols_.p, (const void*)cell_.p, (const void*)anchor_.p, (const void*)gptr_.p,
                          (const void*)gidx_.p, (const void*)ganchor_.p, (const void*)cptr_.p, (const void*)ccol_.p,
                          (const void*)cval_.p, (const void*)liptr_.p, (const void*)licol_.p, (const void*)lival_.p,
                          (const void*)uiptr_.p, (const void*)uicol_.p, (const void*)uival_.p, (const void*)x_.p,
                          (const void*)r_.p, (const void*)c_.p, (const void*)p_.p, (const void*)v_.p,
                          (const void*)s_.p, (const void*)t_.p, (const void*)y_.p, (const void*)z_.p,
                          (const void*)full_.p, (const void*)zfull_.p, (const void*)zp_.p, (const void*)partial_.p,
                          (const void*)state_.p, (const void*)counter_.p})
        key.push_back(reinterpret_cast<uintptr_t>(q));
    for (const TriView* v : {&lview_, &uview_}) {
        const unsigned char* b = reinterpret_cast<const unsigned char*>(v);
        for (size_t i = 0; i < sizeof(TriView); i += sizeof(uintptr_t)) {
            uintptr_t w = 0;
            std::memcpy(&w, b + i, std::min(sizeof(uintptr_t), sizeof(TriView) - i));
            key.push_back(w);
        }
    }
    const int slot = preconditioned ? 1 : 0;
    if (exec_[slot] && key == key_[slot]) return exec_[slot];
    if (exec_[slot]) cudaGraphExecDestroy(exec_[slot]);
    exec_[slot] = nullptr;
    cudaGraph_t graph;
    TPA_CUDA(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle handle;
    TPA_CUDA(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
    alignas(cudaGraphNodeParams) unsigned char cp_storage[sizeof(cudaGraphNodeParams)];
    std::memset(cp_storage, 0, sizeof(cp_storage));
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(cp_storage);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    TPA_CUDA(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    const int before = launches_, ds_before = ds.kernel_launches();
    TPA_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_iteration(ds, f, preconditioned, precision, s, handle, 1);
    cudaGraph_t captured;
    const cudaError_t ce = cudaStreamEndCapture(s, &captured);
    body_launches_[slot] = (launches_ - before);
    launches_ = before;
    ds.add_launches(ds_before - ds.kernel_launches());  // the capture launched nothing
    if (ce != cudaSuccess) {
        cudaGraphDestroy(graph);
        throw Error(2, std::string("graph capture failed: ") + cudaGetErrorString(ce));
    }
    cudaGraphExec_t exec;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) throw Error(2, std::string("graph instantiation failed: ") + cudaGetErrorString(ie));
    exec_[slot] = exec;
    key_[slot] = key;
    return exec;
}

// dst_xi = (L U)^-1 (src_xi / rows_xi - C zp) / cols_xi: the jump block of the
// block preconditioner (rows, cols: D_r, D_c) or of the warm start (ones)
void CmdgfmDevice::jump_apply(const double* src, const double* rows, const double* cols, const double* zp,
                              double* dst, cudaStream_t s) {
    if (inverse_)
        k_cm_jump_inverse<<<1, kIluThreads, 2 * size_t(nx_) * sizeof(double), s>>>(
            int(nx_), np_, src, rows, cptr_.p, ccol_.p, cval_.p, zp, liptr_.p, licol_.p, lival_.p, uiptr_.p, uicol_.p,
            uival_.p, cols, dst);
    else
        k_cm_jump_solve<<<1, kIluThreads, jsmem_, s>>>(int(nx_), np_, src, rows, cptr_.p, ccol_.p, cval_.p, zp,
                                                       lview_, uview_, jstaged_, cols, dst);
    ++launches_;
}

int CmdgfmDevice::bicgstab(DeviceSolver& ds, const CmdgfmInput& in, const CmdgfmFactor& f, bool preconditioned,
                           double rtol, int itmax, cudaStream_t s) {
    const int g = grid_of(n_);
    double* p1 = partial_.p;
    double* st = state_.p;
    double hs[kStateSize];
    auto read = [&] {
        TPA_CUDA(cudaMemcpyAsync(hs, st, sizeof(hs), cudaMemcpyDeviceToHost, s));
        TPA_CUDA(cudaStreamSynchronize(s));
    };
    // x0 = 0, r = p = b (= c_), the shadow residual c = b
    k_cm_init<<<g, kT, 0, s>>>(n_, c_.p, x_.p, r_.p, p_.p, v_.p, p1);
    k_cm_init_fold<<<1, kT, 0, s>>>(p1, g, rtol, itmax, st);
    launches_ += 2;
    read();
    if (int(hs[kFlags]) & (kZeroRhs | kZeroRho | kSolved | kTired)) return 0;
    if (s && !std::getenv("TPAGMG_NO_GRAPH")) {
        // the whole run as one graph launch; the host reads the state at its end
        cudaGraphExec_t exec = loop_graph(ds, f, preconditioned, in.precision, s);
        TPA_CUDA(cudaGraphLaunch(exec, s));
        read();
        launches_ += int(hs[kIter]) * body_launches_[preconditioned ? 1 : 0];
    } else {
        for (;;) {
            enqueue_iteration(ds, f, preconditioned, in.precision, s, cudaGraphConditionalHandle(), 0);
            read();
            if (int(hs[kFlags]) & (kSolved | kTired | kBreakdown)) break;
        }
    }
    TPA_CUDA(cudaGetLastError());
    return int(hs[kIter]);
}

void CmdgfmDevice::solve(DeviceSolver& ds, const CmdgfmInput& in, const CmdgfmFactor& f, double* solution,
                         CmdgfmStats& st) {
    const double eps = 2.220446049250313e-16;
    cudaStream_t s = ds.stream();
    st = CmdgfmStats();
    n_ = in.m.n;
    np_ = in.np;
    nx_ = n_ - np_;
    na_ = in.extra.n;
    ncells_ = ds.ncells();
    launches_ = 0;
    if (nx_ * int64_t(sizeof(double)) > 200 * 1024)
        throw Error(5, "the jump block has more than 25,600 unknowns (its factor solve keeps them in shared memory)");
    cudaEvent_t e0, e1;
    TPA_CUDA(cudaEventCreate(&e0));
    TPA_CUDA(cudaEventCreate(&e1));
    TPA_CUDA(cudaEventRecord(e0, s));
    // the system and the factor
    mptr_.upload(in.m.ptr.data(), in.m.ptr.size(), s);
    mcol_.upload(in.m.col.data(), in.m.col.size(), s);
    mval_.upload(in.m.val.data(), in.m.val.size(), s);
    rhs_.upload(in.rhs.data(), in.rhs.size(), s);
    weight_.upload(in.weight.data(), in.weight.size(), s);
    rows_.upload(in.row_scale.data(), in.row_scale.size(), s);
    cols_.upload(in.col_scale.data(), in.col_scale.size(), s);
    cell_.upload(in.cell.data(), in.cell.size(), s);
    anchor_.upload(in.anchor.data(), in.anchor.size(), s);
    eptr_.upload(in.extra.ptr.data(), in.extra.ptr.size(), s);
    ecol_.upload(in.extra.col.data(), in.extra.col.size(), s);
    eval_.upload(in.extra.val.data(), in.extra.val.size(), s);
    erhs_.upload(in.extra_rhs.data(), in.extra_rhs.size(), s);
    eweight_.upload(in.extra_weight.data(), in.extra_weight.size(), s);
    // anchors and their members (indices increasing) for the reduced scatter
    std::vector<int32_t> anchors(in.anchor.begin(), in.anchor.end());
    std::sort(anchors.begin(), anchors.end());
    anchors.erase(std::unique(anchors.begin(), anchors.end()), anchors.end());
    ngroups_ = int(anchors.size());
    std::vector<int32_t> gptr(static_cast<size_t>(ngroups_) + 1, 0), gidx(static_cast<size_t>(np_));
    for (int64_t i = 0; i < np_; ++i) {
        const int g = int(std::lower_bound(anchors.begin(), anchors.end(), in.anchor[size_t(i)]) - anchors.begin());
        ++gptr[size_t(g) + 1];
    }
    for (int g = 0; g < ngroups_; ++g) gptr[size_t(g) + 1] += gptr[size_t(g)];
    {
        std::vector<int32_t> cur(gptr.begin(), gptr.end() - 1);
        for (int64_t i = 0; i < np_; ++i) {
            const int g = int(std::lower_bound(anchors.begin(), anchors.end(), in.anchor[size_t(i)]) - anchors.begin());
            gidx[size_t(cur[size_t(g)]++)] = int32_t(i);
        }
    }
    anchor1_ = ngroups_ == 1 ? anchors[0] : -1;
    if (!counter_.p) {
        counter_.alloc(1);
        TPA_CUDA(cudaMemsetAsync(counter_.p, 0, sizeof(unsigned), s));
    }
    gptr_.upload(gptr.data(), gptr.size(), s);
    gidx_.upload(gidx.data(), gidx.size(), s);
    ganchor_.upload(anchors.data(), anchors.size(), s);
    cptr_.upload(f.coupling.ptr.data(), f.coupling.ptr.size(), s);
    ccol_.upload(f.coupling.col.data(), f.coupling.col.size(), s);
    cval_.upload(f.coupling.val.data(), f.coupling.val.size(), s);
    if (nx_ > 0) {
        // each factor's rows in solve order, entries contiguous per position: the
        // level schedule, or -- when its levels average fewer than 16 rows --
        // plain row order for one thread
        auto lay_out = [&](const CsrRows& m, const LevelSchedule& sc, bool upper, DevBuf<int32_t>& dptr,
                           DevBuf<int32_t>& dcol, DevBuf<double>& dval, DevBuf<int32_t>& dlev,
                           DevBuf<int32_t>& drows, DevBuf<double>* dinv, TriView& view, size_t& bytes) {
            const int levels = sc.levels();
            const bool seq = double(nx_) < 16.0 * double(std::max(levels, 1));
            std::vector<int32_t> order, lev;
            if (seq) {
                for (int64_t i = 0; i < nx_; ++i) order.push_back(int32_t(upper ? nx_ - 1 - i : i));
                lev = {0, int32_t(nx_)};
            } else {
                order = sc.rows;
                lev = sc.level_ptr;
            }
            std::vector<int32_t> ptr(1, 0), col;
            std::vector<double> val, inv;
            for (int32_t k : order) {
                for (int64_t e = m.ptr[size_t(k)]; e < m.ptr[size_t(k) + 1]; ++e) {
                    col.push_back(m.col[size_t(e)]);
                    val.push_back(m.val[size_t(e)]);
                }
                ptr.push_back(int32_t(col.size()));
                if (upper) inv.push_back(1.0 / f.pivot[size_t(k)]);
            }
            dptr.upload(ptr.data(), ptr.size(), s);
            dcol.upload(col.data(), col.size(), s);
            dval.upload(val.data(), val.size(), s);
            dlev.upload(lev.data(), lev.size(), s);
            drows.upload(order.data(), order.size(), s);
            if (dinv) dinv->upload(inv.data(), inv.size(), s);
            view.nlev = int(lev.size()) - 1;
            view.nnz = int(col.size());
            view.seq = seq ? 1 : 0;
            view.lev = dlev.p;
            view.rows = drows.p;
            view.ptr = dptr.p;
            view.col = dcol.p;
            view.val = dval.p;
            view.inv = dinv ? dinv->p : nullptr;
            bytes = col.size() * 8 + (upper ? size_t(nx_) * 8 : 0) +
                    (lev.size() + size_t(nx_) + size_t(nx_) + 1 + col.size()) * 4 + 8;
            llevels_ = upper ? llevels_ : levels;
            ulevels_ = upper ? levels : ulevels_;
        };
        size_t lb = 0, ub = 0;
        lay_out(f.lower, f.lsched, false, lptr_, lcol_, lval_, lsched_, lrows_, nullptr, lview_, lb);
        lay_out(f.upper, f.usched, true, uptr_, ucol_, uval_, usched_, urows_, &piv_, uview_, ub);
        const size_t full = size_t(nx_) * 8 + lb + ub;
        jstaged_ = full <= size_t(200) * 1024 ? 1 : 0;
        jsmem_ = jstaged_ ? full : size_t(nx_) * 8;
        TPA_CUDA(cudaFuncSetAttribute(k_cm_jump_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(std::max<size_t>(jsmem_, 1))));
        // the inverses, when the host formed them and two vectors fit in shared memory
        // (TPAGMG_CMDGFM_WALK keeps the row walk, to compare the two paths)
        inverse_ = !f.linv.ptr.empty() && 2 * size_t(nx_) * sizeof(double) <= size_t(200) * 1024 &&
                   !std::getenv("TPAGMG_CMDGFM_WALK");
        if (inverse_) {
            liptr_.upload(f.linv.ptr.data(), f.linv.ptr.size(), s);
            licol_.upload(f.linv.col.data(), f.linv.col.size(), s);
            lival_.upload(f.linv.val.data(), f.linv.val.size(), s);
            uiptr_.upload(f.uinv.ptr.data(), f.uinv.ptr.size(), s);
            uicol_.upload(f.uinv.col.data(), f.uinv.col.size(), s);
            uival_.upload(f.uinv.val.data(), f.uinv.val.size(), s);
            TPA_CUDA(cudaFuncSetAttribute(k_cm_jump_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(2 * size_t(nx_) * sizeof(double))));
        }
    }
    for (auto* b : {&sol_, &corr_, &x_, &r_, &c_, &p_, &v_, &s_, &t_, &y_, &z_}) b->alloc(size_t(std::max<int64_t>(n_, 1)));
    full_.alloc(size_t(std::max<int64_t>(ncells_, 1)));
    zfull_.alloc(size_t(std::max<int64_t>(ncells_, 1)));
    zp_.alloc(size_t(std::max<int64_t>(np_, 1)));
    jr_.alloc(size_t(std::max<int64_t>(nx_, 1)));
    partial_.alloc(4 * size_t(kG));
    state_.alloc(kStateSize);
    TPA_CUDA(cudaMemsetAsync(sol_.p, 0, sizeof(double) * size_t(n_), s));
    TPA_CUDA(cudaMemcpyAsync(corr_.p, rhs_.p, sizeof(double) * size_t(n_), cudaMemcpyDeviceToDevice, s));

    const int g = grid_of(n_), ga = grid_of(na_);
    double* p1 = partial_.p;
    double* p2 = partial_.p + kG;
    double* p3 = partial_.p + 2 * kG;
    double* p4 = partial_.p + 3 * kG;
    double hs[kStateSize];
    auto read = [&] {
        TPA_CUDA(cudaMemcpyAsync(hs, state_.p, sizeof(hs), cudaMemcpyDeviceToHost, s));
        TPA_CUDA(cudaStreamSynchronize(s));
    };
    auto defects = [&] {
        k_cm_defects<<<g, kT, 0, s>>>(n_, np_, corr_.p, weight_.p, rows_.p, p1, p2, p3);
        if (na_ > 0)
            k_cm_anchor_defect<<<ga, kT, 0, s>>>(na_, eptr_.p, ecol_.p, eval_.p, erhs_.p, eweight_.p, sol_.p, p4);
        k_cm_defects_fold<<<1, kT, 0, s>>>(p1, p2, p3, g, p4, na_ > 0 ? ga : 0, state_.p);
        launches_ += na_ > 0 ? 3 : 2;
        read();
    };
    auto count = [&](auto launch) {  // a fold of per-block counts
        launch();
        k_cm_sum_fold<<<1, kT, 0, s>>>(p1, g, state_.p + kNorm2);
        launches_ += 2;
        read();
        return hs[kNorm2];
    };
    double rr = 0;
    for (double v : in.rhs) rr += v * v;
    st.initial_residual = std::sqrt(rr);
    const double tol = in.tolerance;
    int iterations = 0;
    if (n_ > 0 && st.initial_residual > 0 && in.warm_start) {
        // `_cmdgfm_initial_solution!` (cmdgfm_projection.jl:1973-2040): zero
        // pressure, then the given previous increment, each with its jumps
        // from the jump factor; the best one that lowers the defect below 0.95
        // of the best so far and the scaled residual norm replaces x = 0
        auto row_defects = [&](const double* res) {
            k_cm_defects<<<g, kT, 0, s>>>(n_, np_, res, weight_.p, rows_.p, p1, p2, p3);
            k_cm_defects_fold<<<1, kT, 0, s>>>(p1, p2, p3, g, p4, 0, state_.p);
            launches_ += 2;
            read();
            const double pd = hs[kPressureDefect], jd = hs[kJumpDefect];
            return std::make_pair((pd != pd || jd != jd) ? NAN : std::max(pd, jd), std::sqrt(hs[kRhsNorm2]));
        };
        if (!ones_.p || ones_.n < size_t(n_)) {
            ones_.alloc(size_t(n_));
            const std::vector<double> one(size_t(n_), 1.0);
            TPA_CUDA(cudaMemcpyAsync(ones_.p, one.data(), sizeof(double) * size_t(n_), cudaMemcpyHostToDevice, s));
            TPA_CUDA(cudaStreamSynchronize(s));
        }
        auto best = row_defects(corr_.p);
        for (int use_previous = 0; use_previous < 2; ++use_previous) {
            TPA_CUDA(cudaMemsetAsync(y_.p, 0, sizeof(double) * size_t(n_), s));
            if (use_previous) {
                if (in.initial.empty()) continue;
                bool any = false, finite = true;
                for (double v : in.initial) {
                    any = any || v != 0.0;
                    finite = finite && std::isfinite(v);
                }
                if (!any || !finite) continue;
                TPA_CUDA(cudaMemcpyAsync(y_.p, in.initial.data(), sizeof(double) * size_t(np_),
                                         cudaMemcpyHostToDevice, s));
            }
            if (nx_ > 0) jump_apply(rhs_.p, ones_.p, ones_.p, y_.p, y_.p, s);
            if (count([&] { k_cm_nonfinite<<<g, kT, 0, s>>>(n_, y_.p, p1); }) != 0.0) continue;
            k_cm_residual<<<g, kT, 0, s>>>(n_, mptr_.p, mcol_.p, mval_.p, rhs_.p, y_.p, t_.p);
            ++launches_;
            const auto cand = row_defects(t_.p);
            if (std::isfinite(cand.first) && std::isfinite(cand.second) && cand.first < 0.95 * best.first &&
                cand.second < best.second) {
                TPA_CUDA(cudaMemcpyAsync(sol_.p, y_.p, sizeof(double) * size_t(n_), cudaMemcpyDeviceToDevice, s));
                best = cand;
                st.initial_guess_used = true;
            }
        }
        k_cm_residual<<<g, kT, 0, s>>>(n_, mptr_.p, mcol_.p, mval_.p, rhs_.p, sol_.p, corr_.p);
        ++launches_;
    }
    if (n_ > 0 && st.initial_residual > 0) {
        while (iterations < in.max_iterations) {
            defects();
            const double pd = hs[kPressureDefect], jd = hs[kJumpDefect], ad = hs[kAnchorDefect];
            const double defect = (pd != pd || jd != jd || ad != ad) ? NAN : std::max(pd, std::max(jd, ad));
            if (!std::isfinite(defect) || defect <= tol) break;
            const double rhs_norm = std::sqrt(hs[kRhsNorm2]);
            if (!std::isfinite(rhs_norm) || rhs_norm == 0.0) break;
            const double requested = std::min(tol, tol / std::max(defect, eps));
            // a tiny correction is normalized before the Krylov run, its scale restored after
            const bool normalize = rhs_norm < 1.0 && rhs_norm * requested < eps;
            const double rhs_scale = normalize ? rhs_norm : 1.0;
            k_cm_scaled_rhs<<<g, kT, 0, s>>>(n_, rows_.p, corr_.p, c_.p, normalize ? 1 : 0, rhs_norm);
            ++launches_;
            int its = bicgstab(ds, in, f, true, requested, in.max_iterations - iterations, s);
            iterations += its;
            ++st.attempts;
            auto nonfinite = [&] {
                return count([&] { k_cm_nonfinite<<<g, kT, 0, s>>>(n_, x_.p, p1); });
            };
            bool finite = nonfinite() == 0.0;
            if (!finite && iterations < in.max_iterations) {
                // the unpreconditioned retry within the remaining budget
                its = bicgstab(ds, in, f, false, requested, in.max_iterations - iterations, s);
                iterations += its;
                ++st.attempts;
                finite = nonfinite() == 0.0;
            }
            if (!finite || its == 0) break;
            const double changed =
                count([&] { k_cm_apply<<<g, kT, 0, s>>>(n_, sol_.p, cols_.p, rhs_scale, x_.p, p1); });
            if (changed == 0.0) break;
            k_cm_residual<<<g, kT, 0, s>>>(n_, mptr_.p, mcol_.p, mval_.p, rhs_.p, sol_.p, corr_.p);
            ++launches_;
        }
    }
    defects();
    st.pressure_defect = hs[kPressureDefect];
    st.jump_defect = hs[kJumpDefect];
    st.anchor_defect = na_ > 0 ? hs[kAnchorDefect] : 0.0;
    st.final_residual = std::sqrt(count([&] { k_cm_dot2<<<g, kT, 0, s>>>(n_, corr_.p, corr_.p, nullptr, nullptr, p1, nullptr); }));
    const double worst = std::max(st.pressure_defect, std::max(st.jump_defect, st.anchor_defect));
    st.converged = std::isfinite(worst) && worst <= tol;
    st.iterations = iterations;
    TPA_CUDA(cudaMemcpyAsync(solution, sol_.p, sizeof(double) * size_t(n_), cudaMemcpyDeviceToHost, s));
    TPA_CUDA(cudaEventRecord(e1, s));
    TPA_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    st.device_ms = ms;
    st.launches = launches_;
    st.inverse = inverse_;
    TPA_CUDA(cudaGetLastError());
}

}  // namespace tpa
