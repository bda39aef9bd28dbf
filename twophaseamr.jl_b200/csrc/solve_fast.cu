// `solve!` around the graph-captured CG loop, with its set-up and checks fused
// into two finest-level passes (default cycle, at most one ungauged component).
//
// The steps are those of src/solvers/multigrid/elliptic_solver.jl:628-675
// (ronaldremmerswaal/TwoPhaseAMR.jl): b = V f with covered cells zeroed, the
// component projection of b (`_project_component_rhs!`, :153-190), the gauge of
// the initial guess, the initial norms and target (`_solve_krylov_with_stats!`,
// :550-612, with the roundoff floor of cycles.jl:108-206), Krylov runs with
// restarts from the true residual (`_run_krylov_reliably!`, :487-526) and the
// final gauge.  `k_prep` folds the three sums the projection and the gauge need;
// `k_pres` applies them and evaluates the residual, its two norms and both
// inputs of the roundoff floor in the same pass.
#include <algorithm>
#include <cmath>
#include <cstdlib>

#include "device.cuh"

namespace tpa {
namespace {

constexpr int kGrid = 1184;  // 8 CTAs on each of 148 SMs
constexpr int kCPrep = 8, kCPres = 9, kCMean = 10;

__device__ __forceinline__ double block_max_all(double v) {
    __shared__ double sh[32];
    __shared__ int nan_seen;
    bool nan = v != v;
    double m = nan ? 0.0 : v;
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (threadIdx.x == 0) nan_seen = 0;
    __syncthreads();
    if (nan) nan_seen = 1;
    if (!lane) sh[wid] = m;
    __syncthreads();
    m = 0;
    if (threadIdx.x < (blockDim.x >> 5)) m = sh[threadIdx.x];
    if (wid == 0)
        for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    __syncthreads();
    return nan_seen ? NAN : m;
}

// Publish N block values (sums where max_mask bit k is 0, maxima where it is 1)
// and fold them in the last block in block order into out[0..N).
template <int N>
__device__ __forceinline__ void publish_fold(const double (&v)[N], unsigned max_mask, double* partial,
                                             unsigned* counter, double* out) {
    __shared__ bool last;
    double b[N];
    for (int k = 0; k < N; ++k) b[k] = (max_mask >> k) & 1 ? block_max_all(v[k]) : block_sum_all(v[k]);
    if (threadIdx.x == 0) {
        for (int k = 0; k < N; ++k) partial[k * gridDim.x + blockIdx.x] = b[k];
        __threadfence();
        const unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int k = 0; k < N; ++k) {
        const double r = (max_mask >> k) & 1 ? fold_partials_max(partial + k * gridDim.x, gridDim.x)
                                             : fold_partials(partial + k * gridDim.x, gridDim.x);
        if (threadIdx.x == 0) out[k] = r;
        __syncthreads();
    }
    if (threadIdx.x == 0) *counter = 0;
}

// b = V f (0 where V = 0), x0 = x_in (0 where V = 0); out = {sum b, sum |b|, sum V x0}.
// vol null: every cell's volume is vol0.
__global__ void k_prep(int n, const double* __restrict__ rhs, const double* __restrict__ xin,
                       const double* __restrict__ vol, double vol0, double* __restrict__ b, double* __restrict__ x0,
                       double* partial, unsigned* counter, double* out) {
    double v[3] = {0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double V = vol ? vol[i] : vol0;
        const double bi = V > 0 ? rhs[i] * V : 0.0;
        const double xi = V > 0 ? xin[i] : 0.0;
        b[i] = bi;
        x0[i] = xi;
        v[0] += bi;
        v[1] += fabs(bi);
        v[2] += V * xi;
    }
    publish_fold<3>(v, 0u, partial, counter, out);
}

// b -= V mb, x = x0 - mx (0 where V = 0), r = b - A x; out = {sum_V r^2 / V,
// max |r| / V, max (|A| |x|) / V, max |b| / V} over cells with V > 0.  A x is
// summed as sum_j a_ij (x_j - x_i) (+ bdiag_i x_i at open sides): the rows
// sum to that conductance (the area-weighted jump maps constants to zero), and
// this form rounds at
// the level of the face fluxes, as the factorized action of elliptic.jl:
// 1125-1180 does, not at the level of a_ii x_i.  The projection step relies on
// it: dt max |div u| after the update equals the final residual over 1/dt^2 to
// a few ulps only when both are evaluated from face differences.
__global__ void k_pres(LevelView<double> A, double* __restrict__ b, const double* __restrict__ x0,
                       double* __restrict__ x, double* __restrict__ r, double mb, double mx, int masked,
                       double* partial, unsigned* counter, double* out) {
    double v[4] = {0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
        const double V = A.vol[i];
        double bi = b[i];
        if (mb != 0.0 && V > 0) {
            bi -= V * mb;
            b[i] = bi;
        }
        const double xi = V > 0 ? x0[i] - mx : 0.0;
        double acc = 0, aacc = 0;
        for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) {
            const int j = A.ci[k];
            const double xj = (!masked || A.vol[j] > 0) ? x0[j] - mx : 0.0;
            acc += A.val[k] * (xj - xi);
            aacc += fabs(A.val[k]) * fabs(xj);
        }
        if (A.bdiag) acc += A.bdiag[i] * xi;  // rows at open sides do not sum to zero
        x[i] = xi;
        const double ri = bi - acc;
        r[i] = ri;
        if (V > 0) {
            v[0] += ri * ri / V;
            const double q = fabs(ri) / V;
            v[1] = (q != q || v[1] != v[1]) ? NAN : fmax(v[1], q);
            v[2] = fmax(v[2], aacc / V);
            v[3] = fmax(v[3], fabs(bi) / V);
        }
    }
    publish_fold<4>(v, 0xEu, partial, counter, out);
}

// k_pres on a constant-coefficient 16x16 finest level (vectorized quads,
// stencil4.cuh): the row is c0 (count x_c - sum of neighbours), evaluated as
// c0 sum (x_c - x_nb) like k_pres; |A| |x| = |c0| (count |x_c| + sum |neighbours|).
__global__ void __launch_bounds__(256) v_pres(SView<double> S, double* __restrict__ b, const double* __restrict__ x0,
                                              double* __restrict__ x, double* __restrict__ r, double mb, double mx,
                                              double* partial, unsigned* counter, double* out) {
    double v[4] = {0, 0, 0, 0};
    const int groups = (S.nblocks + 3) / 4;
    const double* vol = S.vol;
    const double ac0 = fabs(S.c0);
    for (int grp = blockIdx.x; grp < groups; grp += gridDim.x) {
        const QPos p = q_pos(grp);
        const bool valid = p.b < S.nblocks;
        // a level of equal positive volumes needs no per-cell volume loads
        const bool uniform = S.const_vol && S.vol0 > 0;
        const QNb<double> g = q_gather<double>(
            S, p, valid, [&](int c) { return q_ldv(x0 + c); },
            [&](double xv, int c) { return (uniform || vol[c] > 0) ? xv - mx : 0.0; });
        if (!valid) continue;
        const Quad<double> vq = uniform ? Quad<double>{{S.vol0, S.vol0, S.vol0, S.vol0}} : q_ld(vol + p.c);
        Quad<double> bq = q_ldv(b + p.c), rq;
        for (int m = 0; m < 4; ++m) {
            const bool hw = m > 0 || g.hw, he = m < 3 || g.he;
            const double xc = g.x.v[m];
            double nb = 0.0, diff = 0.0;
            int cnt = 0;
            if (hw) {
                const double t = m > 0 ? g.x.v[m - 1] : g.w;
                nb += fabs(t), diff += xc - t, ++cnt;
            }
            if (he) {
                const double t = m < 3 ? g.x.v[m + 1] : g.e;
                nb += fabs(t), diff += xc - t, ++cnt;
            }
            if (g.hs) nb += fabs(g.s.v[m]), diff += xc - g.s.v[m], ++cnt;
            if (g.hn) nb += fabs(g.n.v[m]), diff += xc - g.n.v[m], ++cnt;
            const double aacc = ac0 * (double(cnt) * fabs(xc) + nb);
            const double axm = S.c0 * diff;
            const double V = vq.v[m];
            double bi = bq.v[m];
            if (mb != 0.0 && V > 0) bi -= V * mb;
            bq.v[m] = bi;
            const double ri = bi - axm;
            rq.v[m] = ri;
            if (V > 0) {
                v[0] += ri * ri / V;
                const double q = fabs(ri) / V;
                v[1] = (q != q || v[1] != v[1]) ? NAN : fmax(v[1], q);
                v[2] = fmax(v[2], aacc / V);
                v[3] = fmax(v[3], fabs(bi) / V);
            }
        }
        if (mb != 0.0) q_st(b + p.c, bq);
        q_st(x + p.c, g.x);
        q_st(r + p.c, rq);
    }
    publish_fold<4>(v, 0xEu, partial, counter, out);
}

// out = sum V x; x0 = x (the next k_pres reads x0 and writes x).  vol null:
// every cell's volume is vol0.
__global__ void k_xmean(int n, const double* __restrict__ x, const double* __restrict__ vol, double vol0,
                        double* __restrict__ x0, double* partial, unsigned* counter, double* out) {
    double v[1] = {0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double xi = x[i];
        x0[i] = xi;
        v[0] += (vol ? vol[i] : vol0) * xi;
    }
    publish_fold<1>(v, 0u, partial, counter, out);
}

}  // namespace

void DeviceSolver::solve_fast(const double* rhs, double* x_user, double rtol, double atol, int max_cycles,
                              int compatibility, int precision, SolveStats& st) {
    const double eps = 2.220446049250313e-16;
    DevLevel& L = levels_[0];
    const int n = L.n;
    const LevelView<double>& A = vd_[0];
    const int64_t want = (int64_t(n) + kThreads - 1) / kThreads;
    double* out = spres_.p;
    const double cvol = L.ncomp == 1 ? L.comp_volume[0] : 0.0;
    double vt = 0;  // total volume of cells with V > 0
    for (double v : L.comp_volume) vt += v;
    if (L.ncomp == 0) vt = vol_total_;
    auto read = [&](int count) {
        TPA_CUDA(cudaMemcpyAsync(host_d_, out, size_t(count) * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        TPA_CUDA(cudaStreamSynchronize(stream_));
    };
    cudaEvent_t e0, e1;
    TPA_CUDA(cudaEventCreate(&e0));
    TPA_CUDA(cudaEventCreate(&e1));
    TPA_CUDA(cudaEventRecord(e0, stream_));
    st = SolveStats();

    k_prep<<<fold_grid(k_prep, kThreads, want, kGrid), kThreads, 0, stream_>>>(n, rhs, x_user, L.const_vol ? nullptr : A.vol, L.vol0, b_.p, tmp_.p, spartial_.p, counters_.p + kCPrep,
                                           out);
    ++launches_;
    read(3);
    // a non-finite right-hand side value makes sum |b| non-finite
    if (!std::isfinite(host_d_[1])) throw Error(4, "right-hand side must be finite");
    double mb = 0, mx = 0;
    if (L.ncomp == 1) {
        if (compatibility == 1 && std::fabs(host_d_[0]) > 256 * eps * std::max(1.0, host_d_[1]))
            throw Error(1, "Poisson right-hand side has nonzero volume mean");
        mb = host_d_[0] / cvol;
        mx = host_d_[2] / cvol;
        st.removed_rhs_mean = mb;
        st.removed_max_component_mean = std::fabs(mb);
    }
    struct Norms {
        double l2, linf, floor;
    };
    auto pres = [&](double b_mean, double x_mean) {
        if (sdev_[0].vec) {
            const int groups = (sd_[0].nblocks + 3) / 4;
            v_pres<<<fold_grid(v_pres, 256, groups, kGrid), 256, 0, stream_>>>(
                sd_[0], b_.p, tmp_.p, xw_.p, r_.p, b_mean, x_mean, spartial_.p, counters_.p + kCPres, out);
        } else {
            k_pres<<<fold_grid(k_pres, kThreads, want, kGrid), kThreads, 0, stream_>>>(
                A, b_.p, tmp_.p, xw_.p, r_.p, b_mean, x_mean, L.any_void ? 1 : 0, spartial_.p, counters_.p + kCPres,
                out);
        }
        ++launches_;
        read(4);
        Norms nm;
        nm.l2 = vt > 0 ? std::sqrt(host_d_[0] / vt) : 0.0;
        nm.linf = host_d_[1];
        nm.floor = 128 * eps * std::max(1.0, std::max(host_d_[2], host_d_[3]));
        return nm;
    };
    const Norms init = pres(mb, mx);
    const double target = std::max(atol, std::max(rtol * std::max(init.linf, eps), init.floor));
    auto guarded = [&](double cur, double fl) {
        if (!(std::isfinite(init.linf) && std::isfinite(cur) && target < cur && cur < init.linf)) return target;
        return (std::isfinite(fl) && fl < init.linf / 100) ? std::max(target, fl) : target;
    };
    Norms fin = init;
    int total = 0;
    if (init.linf > target) {
        while (total < max_cycles) {
            int niter = 0, flags = 0;
            // precision 2, FP64 iterative refinement: each run is a CG on the
            // correction with FP32 r, directions and Ap (x and every inner
            // product stay FP64), started from the FP32 rounding of the true
            // residual and stopped at a fixed reduction of it or at the target;
            // its recurrence residual follows the true one to about the FP32
            // unit roundoff per iteration
            const double inner = precision == 2 ? std::max(target, ir_eta_ * fin.linf) : target;
            cg_fused(precision, inner, max_cycles - total, niter, flags);
            total += niter;
            // gauge of the iterate, then the true residual and its norms
            k_xmean<<<fold_grid(k_xmean, kThreads, want, kGrid), kThreads, 0, stream_>>>(n, xw_.p, L.const_vol ? nullptr : A.vol, L.vol0, tmp_.p, spartial_.p, counters_.p + kCMean,
                                                    out);
            ++launches_;
            double xm = 0;
            if (L.ncomp == 1) {
                read(1);
                xm = host_d_[0] / cvol;
            }
            fin = pres(0.0, xm);
            ++st.restarts;
            const double eff = guarded(fin.linf, fin.floor);
            if (fin.linf <= eff) break;
            if (!std::isfinite(fin.linf) || niter == 0) break;
        }
    }
    check_barrier();
    const double tfinal = guarded(fin.linf, fin.floor);
    TPA_CUDA(cudaMemcpyAsync(x_user, xw_.p, sizeof(double) * size_t(n), cudaMemcpyDeviceToDevice, stream_));
    TPA_CUDA(cudaEventRecord(e1, stream_));
    TPA_CUDA(cudaEventSynchronize(e1));
    TPA_CUDA(cudaGetLastError());
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    st.cycles = total;
    st.converged = std::isfinite(fin.linf) && std::isfinite(tfinal) && fin.linf <= tfinal;
    st.initial_l2 = init.l2;
    st.initial_linf = init.linf;
    st.final_l2 = fin.l2;
    st.final_linf = fin.linf;
    st.target_linf = tfinal;
    st.residual_scale = std::max(init.linf, eps);
    st.ms_total = ms;
}

}  // namespace tpa
