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

// full[cell_i] = src_i / rows_i (the reduced right-hand side scattered)
__global__ void k_cm_scatter(int64_t np, const double* __restrict__ src, const double* __restrict__ rows,
                             const int32_t* __restrict__ cell, double* __restrict__ full) {
    CM_LOOP(i, np) full[cell[i]] = src[i] / rows[i];
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

// jr_f = src_(np+f) / rows_(np+f) - sum_c C[f,c] zp_c
__global__ void k_cm_jump_rhs(int64_t nx, int64_t np, const double* __restrict__ src, const double* __restrict__ rows,
                              const int64_t* __restrict__ cptr, const int32_t* __restrict__ ccol,
                              const double* __restrict__ cval, const double* __restrict__ zp,
                              double* __restrict__ jr) {
    CM_LOOP(f, nx) {
        double acc = 0;
        for (int64_t e = cptr[f]; e < cptr[f + 1]; ++e) acc += cval[e] * zp[ccol[e]];
        jr[f] = src[np + f] / rows[np + f] - acc;
    }
}

// One triangular solve of the jump block's factor in one CTA, rows in the
// order of a level schedule: position i holds row rows[i], its entries
// (col, val)[ptr[i] .. ptr[i+1]) in column order and, for U, its pivot
// piv[i]; the rows of level v are positions lev[v] .. lev[v+1] and depend
// only on earlier levels.  The vector lives in shared memory and, when
// `staged`, so does the whole schedule (it is read once per solve).  A thin
// schedule (few rows per level) runs in the first warp alone, with a warp
// barrier between levels instead of a CTA barrier.  Upper: x = U^-1 in,
// written as dst[np + k] = x_k / cols[np + k]; else y = L^-1 in (unit
// diagonal) into out.
template <bool Upper>
__global__ void __launch_bounds__(kIluThreads)
    k_cm_trisolve(int nx, int nlev, const int32_t* __restrict__ glev, const int32_t* __restrict__ grows,
                  const int32_t* __restrict__ gptr, const int32_t* __restrict__ gcol, const double* __restrict__ gval,
                  const double* __restrict__ gpiv, int staged, int thin, const double* __restrict__ in,
                  double* __restrict__ out, int64_t np, const double* __restrict__ cols) {
    extern __shared__ double sm[];
    double* y = sm;
    const int nnz = gptr[nx];
    const double* val = gval;
    const double* piv = gpiv;
    const int32_t *lev = glev, *rows = grows, *ptr = gptr, *col = gcol;
    for (int f = threadIdx.x; f < nx; f += blockDim.x) y[f] = in[f];
    if (staged) {
        double* sval = y + nx;
        double* spiv = sval + nnz;
        int32_t* slev = reinterpret_cast<int32_t*>(spiv + (Upper ? nx : 0));
        int32_t* srows = slev + nlev + 1;
        int32_t* sptr = srows + nx;
        int32_t* scol = sptr + nx + 1;
        for (int e = threadIdx.x; e < nnz; e += blockDim.x) {
            sval[e] = gval[e];
            scol[e] = gcol[e];
        }
        for (int i = threadIdx.x; i < nx; i += blockDim.x) {
            srows[i] = grows[i];
            if (Upper) spiv[i] = gpiv[i];
        }
        for (int i = threadIdx.x; i <= nx; i += blockDim.x) sptr[i] = gptr[i];
        for (int i = threadIdx.x; i <= nlev; i += blockDim.x) slev[i] = glev[i];
        val = sval;
        piv = spiv;
        lev = slev;
        rows = srows;
        ptr = sptr;
        col = scol;
    }
    __syncthreads();
    auto row = [&](int i) {
        const int k = rows[i];
        double acc = y[k];
        for (int e = ptr[i]; e < ptr[i + 1]; ++e) acc -= val[e] * y[col[e]];
        y[k] = Upper ? acc / piv[i] : acc;
    };
    if (thin) {
        if (threadIdx.x < 32) {
            for (int v = 0; v < nlev; ++v) {
                for (int i = lev[v] + int(threadIdx.x); i < lev[v + 1]; i += 32) row(i);
                __syncwarp();
            }
        }
    } else {
        for (int v = 0; v < nlev; ++v) {
            for (int i = lev[v] + int(threadIdx.x); i < lev[v + 1]; i += blockDim.x) row(i);
            __syncthreads();
        }
    }
    __syncthreads();
    for (int f = threadIdx.x; f < nx; f += blockDim.x) {
        if (Upper) out[np + f] = y[f] / cols[np + f];
        else out[f] = y[f];
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
__global__ void k_cm_rho(const double* p1, const double* p2, int count, double* st) {
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
        k_cm_scatter<<<grid_of(np_), kT, 0, s>>>(np_, src, rows_.p, cell_.p, full_.p);
        k_cm_anchor<<<ngroups_, 1024, 0, s>>>(gptr_.p, gidx_.p, ganchor_.p, src, rows_.p, full_.p);
        launches_ += 2;
        const int before = ds.kernel_launches();
        ds.vcycle(full_.p, zfull_.p, precision);
        launches_ += ds.kernel_launches() - before;
        k_cm_gather<<<grid_of(np_), kT, 0, s>>>(np_, zfull_.p, cell_.p, anchor_.p, cols_.p, zp_.p, dst);
        ++launches_;
    }
    if (nx_ > 0) {
        k_cm_jump_rhs<<<grid_of(nx_), kT, 0, s>>>(nx_, np_, src, rows_.p, cptr_.p, ccol_.p, cval_.p, zp_.p, jr_.p);
        k_cm_trisolve<false><<<1, kIluThreads, lsmem_, s>>>(int(nx_), llevels_, lsched_.p, lrows_.p, lptr_.p, lcol_.p,
                                                            lval_.p, nullptr, lstaged_, lthin_, jr_.p, zp2_.p, 0,
                                                            nullptr);
        k_cm_trisolve<true><<<1, kIluThreads, usmem_, s>>>(int(nx_), ulevels_, usched_.p, urows_.p, uptr_.p, ucol_.p,
                                                           uval_.p, piv_.p, ustaged_, uthin_, zp2_.p, dst, np_,
                                                           cols_.p);
        launches_ += 3;
    }
    (void)f;
}

int CmdgfmDevice::bicgstab(DeviceSolver& ds, const CmdgfmInput& in, const CmdgfmFactor& f, bool preconditioned,
                           double rtol, int itmax, cudaStream_t s) {
    const int g = grid_of(n_);
    double* p1 = partial_.p;
    double* p2 = partial_.p + kG;
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
    for (;;) {
        const double* y = p_.p;
        if (preconditioned) {
            precondition(ds, f, p_.p, y_.p, in.precision, s);
            y = y_.p;
        }
        spmv(y, v_.p, 1, s);
        k_cm_dot2<<<g, kT, 0, s>>>(n_, c_.p, v_.p, nullptr, nullptr, p1, nullptr);
        k_cm_alpha<<<1, kT, 0, s>>>(p1, g, st);
        k_cm_update1<<<g, kT, 0, s>>>(n_, r_.p, v_.p, y, s_.p, x_.p, st);
        launches_ += 3;
        const double* z = s_.p;
        if (preconditioned) {
            precondition(ds, f, s_.p, z_.p, in.precision, s);
            z = z_.p;
        }
        spmv(z, t_.p, 1, s);
        k_cm_dot2<<<g, kT, 0, s>>>(n_, t_.p, s_.p, t_.p, t_.p, p1, p2);
        k_cm_omega<<<1, kT, 0, s>>>(p1, p2, g, st);
        k_cm_update2<<<g, kT, 0, s>>>(n_, s_.p, t_.p, z, c_.p, x_.p, r_.p, st, p1, p2);
        k_cm_rho<<<1, kT, 0, s>>>(p1, p2, g, st);
        k_cm_pupdate<<<g, kT, 0, s>>>(n_, r_.p, v_.p, p_.p, st);
        launches_ += 5;
        read();
        if (int(hs[kFlags]) & (kSolved | kTired | kBreakdown)) break;
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
    gptr_.upload(gptr.data(), gptr.size(), s);
    gidx_.upload(gidx.data(), gidx.size(), s);
    ganchor_.upload(anchors.data(), anchors.size(), s);
    cptr_.upload(f.coupling.ptr.data(), f.coupling.ptr.size(), s);
    ccol_.upload(f.coupling.col.data(), f.coupling.col.size(), s);
    cval_.upload(f.coupling.val.data(), f.coupling.val.size(), s);
    if (nx_ > 0) {
        // each factor's rows in schedule order, entries contiguous per position
        auto lay_out = [&](const CsrRows& m, const LevelSchedule& sc, const std::vector<double>* pv,
                           DevBuf<int32_t>& dptr, DevBuf<int32_t>& dcol, DevBuf<double>& dval,
                           DevBuf<int32_t>& dlev, DevBuf<int32_t>& drows, DevBuf<double>* dpiv, size_t& smem,
                           int& staged, int& thin, int& levels) {
            std::vector<int32_t> ptr(1, 0), col;
            std::vector<double> val, piv;
            for (int32_t k : sc.rows) {
                for (int64_t e = m.ptr[size_t(k)]; e < m.ptr[size_t(k) + 1]; ++e) {
                    col.push_back(m.col[size_t(e)]);
                    val.push_back(m.val[size_t(e)]);
                }
                ptr.push_back(int32_t(col.size()));
                if (pv) piv.push_back((*pv)[size_t(k)]);
            }
            dptr.upload(ptr.data(), ptr.size(), s);
            dcol.upload(col.data(), col.size(), s);
            dval.upload(val.data(), val.size(), s);
            dlev.upload(sc.level_ptr.data(), sc.level_ptr.size(), s);
            drows.upload(sc.rows.data(), sc.rows.size(), s);
            if (dpiv) dpiv->upload(piv.data(), piv.size(), s);
            levels = sc.levels();
            thin = double(nx_) < 64.0 * double(std::max(levels, 1)) ? 1 : 0;
            const size_t nnz = col.size();
            const size_t full = size_t(nx_) * 8 + nnz * 8 + (pv ? size_t(nx_) * 8 : 0) +
                                (size_t(levels) + 1 + size_t(nx_) + size_t(nx_) + 1 + nnz) * 4;
            staged = full <= size_t(200) * 1024 ? 1 : 0;
            smem = staged ? full : size_t(nx_) * 8;
        };
        lay_out(f.lower, f.lsched, nullptr, lptr_, lcol_, lval_, lsched_, lrows_, nullptr, lsmem_, lstaged_, lthin_,
                llevels_);
        lay_out(f.upper, f.usched, &f.pivot, uptr_, ucol_, uval_, usched_, urows_, &piv_, usmem_, ustaged_, uthin_,
                ulevels_);
        TPA_CUDA(cudaFuncSetAttribute(k_cm_trisolve<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(std::max<size_t>(lsmem_, 1))));
        TPA_CUDA(cudaFuncSetAttribute(k_cm_trisolve<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(std::max<size_t>(usmem_, 1))));
    }
    for (auto* b : {&sol_, &corr_, &x_, &r_, &c_, &p_, &v_, &s_, &t_, &y_, &z_}) b->alloc(size_t(std::max<int64_t>(n_, 1)));
    full_.alloc(size_t(std::max<int64_t>(ncells_, 1)));
    zfull_.alloc(size_t(std::max<int64_t>(ncells_, 1)));
    zp_.alloc(size_t(std::max<int64_t>(np_, 1)));
    jr_.alloc(size_t(std::max<int64_t>(nx_, 1)));
    zp2_.alloc(size_t(std::max<int64_t>(nx_, 1)));
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
    TPA_CUDA(cudaGetLastError());
}

}  // namespace tpa
