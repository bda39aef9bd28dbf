// B200 kernels and the device solve of the tree-GMG-preconditioned PCG.
//
// Device counterpart of (ronaldremmerswaal/TwoPhaseAMR.jl):
//   src/solvers/multigrid/cycles.jl:8-77       damped-Jacobi smoothing and the V-cycle
//   src/solvers/multigrid/hierarchy.jl:208-246 prolongation / restriction with
//                                              P = (I - wt Dt^-1 A) P_tent, applied
//                                              matrix-free: P xc = e - wt Dt^-1 A e with
//                                              e = P_tent xc, and P' r = P_tent'(r - wt A Dt^-1 r)
//   src/solvers/multigrid/hierarchy.jl:316-343 component projections
//   src/solvers/multigrid/elliptic_solver.jl:369-675  PCG driver, restarts, stats
//
// The per-sweep component-mean removal of `_smooth!` is folded into one removal
// at the end of the finest level: the level operators annihilate constants and
// P preserves them, so a constant shift of any level iterate changes neither
// the residuals nor the finest-level result after its mean is removed.
//
// Reductions run on a fixed grid (kReduceBlocks) and fold their partials in a
// fixed order, so every result is bitwise repeatable.
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "device.cuh"

namespace tpa {
namespace {

inline int grid_for(int64_t n) {
    int64_t g = (n + kThreads - 1) / kThreads;
    return int(g < 1 ? 1 : g);
}

template <typename T>
__device__ __forceinline__ T row_dot(const int* __restrict__ rp, const int* __restrict__ ci,
                                     const T* __restrict__ v, const T* __restrict__ x, int i) {
    T acc = T(0);
    for (int k = rp[i]; k < rp[i + 1]; ++k) acc += v[k] * x[ci[k]];
    return acc;
}

// A x as sum_j a_ij (x_j - x_i).  Every row of the operator sums to zero (the
// area-weighted jump maps constants to zero and no side is open), so this is
// A x in exact arithmetic; in floating point its rounding scales with the
// differences x_j - x_i, as in the factorized face-flux action (elliptic.jl:
// 1125-1180), rather than with a_ii x_i.  True residuals use it.
__device__ __forceinline__ double row_diff(const int* __restrict__ rp, const int* __restrict__ ci,
                                           const double* __restrict__ v, const double* __restrict__ x, int i) {
    const double xi = x[i];
    double acc = 0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) acc += v[k] * (x[ci[k]] - xi);
    return acc;
}

template <typename T>
__global__ void k_spmv(int n, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ v,
                       const T* __restrict__ x, T* __restrict__ y) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = row_dot(rp, ci, v, x, i);
}

template <typename T>
__global__ void k_jacobi_first(int n, const T* __restrict__ b, const T* __restrict__ dinv, T w, T* __restrict__ x) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = w * dinv[i] * b[i];
}

template <typename T>
__global__ void k_jacobi(int n, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ v,
                         const T* __restrict__ b, const T* __restrict__ dinv, T w, const T* __restrict__ xin,
                         T* __restrict__ xout) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) xout[i] = xin[i] + w * dinv[i] * (b[i] - row_dot(rp, ci, v, xin, i));
}

// red-black half-sweep: cells of colour c updated from xin, the others copied
template <typename T>
__global__ void k_rb_sweep(int n, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ v,
                           const T* __restrict__ b, const T* __restrict__ dinv, const unsigned char* __restrict__ col,
                           int c, T w, const T* __restrict__ xin, T* __restrict__ xout) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) xout[i] = col[i] == c ? xin[i] + w * dinv[i] * (b[i] - row_dot(rp, ci, v, xin, i)) : xin[i];
}

template <typename T>
__global__ void k_residual(int n, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ v,
                           const T* __restrict__ b, const T* __restrict__ x, const T* __restrict__ tinv,
                           T* __restrict__ r, T* __restrict__ s) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        T ri = b[i] - row_dot(rp, ci, v, x, i);
        r[i] = ri;
        s[i] = tinv[i] * ri;
    }
}

// bc[J] = sum over fine children i of J (increasing i) of r_i - tw (A s)_i
template <typename T>
__global__ void k_restrict(int nc, const int* __restrict__ cptr, const int* __restrict__ child,
                           const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ v,
                           const T* __restrict__ r, const T* __restrict__ s, T tw, T* __restrict__ bc) {
    int J = blockIdx.x * blockDim.x + threadIdx.x;
    if (J >= nc) return;
    T acc = T(0);
    for (int k = cptr[J]; k < cptr[J + 1]; ++k) {
        int i = child[k];
        acc += r[i] - tw * row_dot(rp, ci, v, s, i);
    }
    bc[J] = acc;
}

// x_i += e_i - tw Dt^-1_i (A e)_i, e = xc[owner(.)]
template <typename T>
__global__ void k_prolong(int n, const int* __restrict__ rp, const int* __restrict__ ci, const T* __restrict__ v,
                          const int* __restrict__ owner, const T* __restrict__ xc, const T* __restrict__ tinv, T tw,
                          T* __restrict__ x) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T ae = T(0);
    for (int k = rp[i]; k < rp[i + 1]; ++k) ae += v[k] * xc[owner[ci[k]]];
    x[i] += xc[owner[i]] - tw * tinv[i] * ae;
}

// x = G b, one warp per row (FP64 dense coarsest solve)
__global__ void k_coarse(int n, const double* __restrict__ G, const double* __restrict__ b, double* __restrict__ x) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double* row = G + size_t(warp) * n;
    double acc = 0;
    for (int k = lane; k < n; k += 32) acc += row[k] * b[k];
    for (int o = 16; o; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (!lane) x[warp] = acc;
}

template <typename S, typename D>
__global__ void k_convert(int n, const S* __restrict__ s, D* __restrict__ d) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] = D(s[i]);
}

template <typename T>
__global__ void k_fill(int n, T* __restrict__ d, T v) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] = v;
}

// ---- deterministic reductions -------------------------------------------------

__device__ __forceinline__ double block_sum(double v) {
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

__device__ __forceinline__ double block_max(double v) {
    __shared__ double sh[32];
    for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (!lane) sh[wid] = v;
    __syncthreads();
    v = 0;
    if (threadIdx.x < (blockDim.x >> 5)) v = sh[threadIdx.x];
    if (wid == 0)
        for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// mode 0: sum v, 1: sum w*v, 2: sum |v|; restricted to slot == s (slot may be null)
template <typename T>
__global__ void k_slot_sum(int n, const T* __restrict__ v, const T* __restrict__ w, const int* __restrict__ slot,
                           int s, int mode, double* __restrict__ partial) {
    double acc = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (slot && slot[i] != s) continue;
        double x = double(v[i]);
        acc += mode == 0 ? x : mode == 1 ? double(w[i]) * x : fabs(x);
    }
    acc = block_sum(acc);
    if (!threadIdx.x) partial[blockIdx.x] = acc;
}

__global__ void k_dot(int n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ partial) {
    double acc = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc += a[i] * b[i];
    acc = block_sum(acc);
    if (!threadIdx.x) partial[blockIdx.x] = acc;
}

// max |r_i| / V_i over V_i > 0 (NaN propagates)
__global__ void k_strong_max(int n, const double* __restrict__ r, const double* __restrict__ vol,
                             double* __restrict__ partial) {
    double m = 0;
    bool nan = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double V = vol[i];
        if (!(V > 0)) continue;
        double q = fabs(r[i]) / V;
        if (q != q) nan = true;
        m = fmax(m, q);
    }
    m = block_max(m);
    __shared__ int any_nan;
    if (!threadIdx.x) any_nan = 0;
    __syncthreads();
    if (nan) any_nan = 1;
    __syncthreads();
    if (!threadIdx.x) partial[blockIdx.x] = any_nan ? NAN : m;
}

// sum of V (r/V)^2 over V > 0 and sum of V
__global__ void k_l2_terms(int n, const double* __restrict__ r, const double* __restrict__ vol,
                           double* __restrict__ partial) {
    double a = 0, bsum = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double V = vol[i];
        if (!(V > 0)) continue;
        double s = r[i] / V;
        a += V * s * s;
        bsum += V;
    }
    a = block_sum(a);
    bsum = block_sum(bsum);
    if (!threadIdx.x) {
        partial[blockIdx.x] = a;
        partial[gridDim.x + blockIdx.x] = bsum;
    }
}

__global__ void k_fold_sum(const double* __restrict__ partial, int np, double* __restrict__ out) {
    double acc = 0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) acc += partial[i];
    acc = block_sum(acc);
    if (!threadIdx.x) *out = acc;
}

__global__ void k_fold_max(const double* __restrict__ partial, int np, double* __restrict__ out) {
    double m = 0;
    bool nan = false;
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
        double q = partial[i];
        if (q != q) nan = true;
        m = fmax(m, q);
    }
    m = block_max(m);
    __shared__ int any_nan;
    if (!threadIdx.x) any_nan = 0;
    __syncthreads();
    if (nan) any_nan = 1;
    __syncthreads();
    if (!threadIdx.x) *out = any_nan ? NAN : m;
}

// v -= (vol ? vol_i : 1) * sum / cvol on cells of slot s
template <typename T>
__global__ void k_sub_scaled(int n, T* __restrict__ v, const T* __restrict__ vol, const int* __restrict__ slot, int s,
                             const double* __restrict__ sum, double cvol) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (slot && slot[i] != s)) return;
    double mean = *sum / cvol;
    v[i] -= T(vol ? double(vol[i]) * mean : mean);
}

// ---- PCG kernels (FP64, finest level) -------------------------------------------

__global__ void k_scale_rhs(int n, const double* __restrict__ rhs, const double* __restrict__ vol,
                            double* __restrict__ b, double* __restrict__ x) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double V = vol[i];
    if (V == 0) {
        b[i] = 0;
        x[i] = 0;
    } else {
        b[i] = rhs[i] * V;
    }
}

__global__ void k_residual64(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                             const double* __restrict__ b, const double* __restrict__ x, double* __restrict__ r,
                             const double* __restrict__ bdiag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = b[i] - (row_diff(rp, ci, v, x, i) + (bdiag ? bdiag[i] * x[i] : 0.0));
}

__global__ void k_abs_spmv(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                           const double* __restrict__ x, double* __restrict__ y) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc = 0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) acc += fabs(v[k]) * fabs(x[ci[k]]);
    y[i] = acc;
}

// Ap = A p, partial p'Ap
__global__ void k_cg_ap(int n, const int* __restrict__ rp, const int* __restrict__ ci, const double* __restrict__ v,
                        const double* __restrict__ p, double* __restrict__ ap, double* __restrict__ partial) {
    double acc = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double y = row_dot(rp, ci, v, p, i);
        ap[i] = y;
        acc += p[i] * y;
    }
    acc = block_sum(acc);
    if (!threadIdx.x) partial[blockIdx.x] = acc;
}

// alpha = gamma / p'Ap with the zero-curvature guard of Krylov.jl's cg!
__global__ void k_cg_alpha(const double* __restrict__ partial, int np, CgScalars* sc) {
    double acc = 0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) acc += partial[i];
    acc = block_sum(acc);
    if (threadIdx.x) return;
    sc->pAp = acc;
    const double eps = 2.220446049250313e-16;
    if (acc <= eps * sc->pnorm2 && fabs(acc) <= eps * sc->pnorm2) {
        sc->flags |= 2;
        sc->alpha = 0;
    } else {
        sc->alpha = sc->gamma / acc;
    }
}

// x += alpha p, r -= alpha Ap, partial strong max of r
__global__ void k_cg_update(int n, double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                            const double* __restrict__ ap, const double* __restrict__ vol, const CgScalars* sc,
                            double* __restrict__ partial) {
    const double alpha = sc->alpha;
    const bool skip = sc->flags & 2;
    double m = 0;
    bool nan = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double ri = r[i];
        if (!skip) {
            x[i] += alpha * p[i];
            ri -= alpha * ap[i];
            r[i] = ri;
        }
        double V = vol[i];
        if (V > 0) {
            double q = fabs(ri) / V;
            if (q != q) nan = true;
            m = fmax(m, q);
        }
    }
    m = block_max(m);
    __shared__ int any_nan;
    if (!threadIdx.x) any_nan = 0;
    __syncthreads();
    if (nan) any_nan = 1;
    __syncthreads();
    if (!threadIdx.x) partial[blockIdx.x] = any_nan ? NAN : m;
}

// gamma_next = r'z, stopping tests, beta; partial[0..np) holds r'z partials,
// partial[np..2np) the strong-max partials of k_cg_update.
__global__ void k_cg_beta(const double* __restrict__ partial, int np, CgScalars* sc) {
    double acc = 0, m = 0;
    bool nan = false;
    for (int i = threadIdx.x; i < np; i += blockDim.x) {
        acc += partial[i];
        double q = partial[np + i];
        if (q != q) nan = true;
        m = fmax(m, q);
    }
    acc = block_sum(acc);
    m = block_max(m);
    __shared__ int any_nan;
    if (!threadIdx.x) any_nan = 0;
    __syncthreads();
    if (nan) any_nan = 1;
    __syncthreads();
    if (threadIdx.x) return;
    if (sc->flags & 2) return;
    sc->strong_max = any_nan ? NAN : m;
    double gn = acc;
    sc->gamma_next = gn;
    double rnorm = sqrt(gn);
    sc->rnorm = rnorm;
    bool solved = (rnorm + 1.0 <= 1.0);
    if (!solved) {
        double beta = gn / sc->gamma;
        sc->beta = beta;
        sc->pnorm2 = gn + beta * beta * sc->pnorm2;
        sc->gamma = gn;
    } else {
        sc->flags |= 4;
    }
    sc->iter += 1;
    if (sc->strong_max <= sc->target) sc->flags |= 1;
}

__global__ void k_cg_p(int n, double* __restrict__ p, const double* __restrict__ z, const CgScalars* sc) {
    if (sc->flags & 6) return;
    const double beta = sc->beta;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = z[i] + beta * p[i];
}

__global__ void k_cg_init(const double* __restrict__ partial, int np, CgScalars* sc, double target) {
    double acc = 0;
    for (int i = threadIdx.x; i < np; i += blockDim.x) acc += partial[i];
    acc = block_sum(acc);
    if (threadIdx.x) return;
    sc->gamma = acc;
    sc->pnorm2 = acc;
    sc->rnorm = sqrt(acc);
    sc->target = target;
    sc->flags = acc == 0 ? 8 : 0;
    sc->iter = 0;
}

}  // namespace

// ---------------------------------------------------------------------------------

DeviceSolver::DeviceSolver(int device) : device_(device) {
    TPA_CUDA(cudaSetDevice(device));
    TPA_CUDA(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking));
    stream_ = own_stream_;
    TPA_CUDA(cudaMallocHost(&host_sc_, sizeof(CgScalars)));
    TPA_CUDA(cudaMallocHost(&host_d_, 64 * sizeof(double)));
    partial_.alloc(static_cast<size_t>(4 * kReduceBlocks));
    sc_.alloc(1);
    sums_.alloc(64);
}

DeviceSolver::~DeviceSolver() {
    cudaSetDevice(device_);
    if (stream_) cudaStreamSynchronize(stream_);
    destroy_graphs();
    levels_.clear();
    if (host_sc_) cudaFreeHost(host_sc_);
    if (host_d_) cudaFreeHost(host_d_);
    if (rstage_) cudaFreeHost(rstage_);
    if (own_stream_) cudaStreamDestroy(own_stream_);
}

template <> DevLevelT<double>& DeviceSolver::lv<double>(int l) { return levels_[size_t(l)].d; }
template <> DevLevelT<float>& DeviceSolver::lv<float>(int l) { return levels_[size_t(l)].f; }

int resident_ctas(const void* fn, int block, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, size_t, int>, int> cache;
    int dev = 0;
    TPA_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_tuple(fn, block, smem, dev);
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int occ = 0, sms = 0;
    TPA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, block, smem));
    TPA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int r = std::max(1, occ) * std::max(1, sms);
    cache.emplace(key, r);
    return r;
}

// Red-black colouring of a level (the reference smooths with damped Jacobi and
// has no colouring): colour (I + J) mod 2 of every cell, (I, J) its lattice
// coordinates at its own block's refinement level; 0 red, 1 black.
std::vector<unsigned char> red_black_colours(const Mesh& m) {
    const int nx = m.bs[0], ny = m.bs[1];
    std::vector<unsigned char> out(static_cast<size_t>(m.ncells()));
    for (int64_t b = 0; b < m.nblocks(); ++b) {
        const int64_t bi = key_i(m.keys[size_t(b)]) * nx, bj = key_j(m.keys[size_t(b)]) * ny;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i)
                out[size_t(b * nx * ny + j * nx + i)] = static_cast<unsigned char>((bi + i + bj + j) & 1);
    }
    return out;
}

// Weight of a red-black half-sweep: the `_jacobi_weight!` rule min(1, 4/(3 b)),
// b = max_i sum_{j of i's colour} |a_ij| / a_ii (rows with a_ii > 0); weight 1
// for an exact two-colouring (b = 1) or without a bound.
double red_black_weight(const Csr& A, const std::vector<unsigned char>& col) {
    double bound = 0.0;
    for (int64_t r = 0; r < A.n; ++r) {
        double d = 0.0, rs = 0.0;
        for (int64_t k = A.ptr[size_t(r)]; k < A.ptr[size_t(r + 1)]; ++k) {
            const int32_t c = A.col[size_t(k)];
            if (c == r) d = A.val[size_t(k)];
            if (col[size_t(c)] == col[size_t(r)]) rs += std::fabs(A.val[size_t(k)]);
        }
        if (d > 0) bound = std::max(bound, rs / d);
    }
    return bound == 0.0 ? 1.0 : std::min(1.0, 4.0 / (3.0 * bound));
}

void DeviceSolver::upload(const Hierarchy& h) {
    TPA_CUDA(cudaSetDevice(device_));
    TPA_CUDA(cudaStreamSynchronize(stream_));
    rl_ready_ = false;  // the refresh term lists belong to the previous topology
    rl_.clear();
    levels_.clear();
    levels_.resize(h.levels.size());
    pre_ = h.opts.pre_sweeps;
    post_ = h.opts.post_sweeps;
    rb_ = h.opts.smoother == 1;
    for (size_t l = 0; l < h.levels.size(); ++l) {
        const HostLevel& hl = h.levels[l];
        DevLevel& d = levels_[l];
        const Csr& A = hl.op.A;
        d.n = int(A.n);
        d.nnz = A.ptr.back();
        if (A.n > INT32_MAX || d.nnz > INT32_MAX) throw Error(5, "level exceeds 32-bit indexing");
        std::vector<int> rp(A.ptr.begin(), A.ptr.end());
        d.rowptr.upload(rp.data(), rp.size(), stream_);
        d.col.upload(A.col.data(), A.col.size(), stream_);
        d.d.val.upload(A.val.data(), A.val.size(), stream_);
        std::vector<float> fv(A.val.begin(), A.val.end());
        d.f.val.upload(fv.data(), fv.size(), stream_);
        d.d.dinv.upload(hl.inv_diag.data(), hl.inv_diag.size(), stream_);
        std::vector<float> fd(hl.inv_diag.begin(), hl.inv_diag.end());
        d.f.dinv.upload(fd.data(), fd.size(), stream_);
        d.d.vol.upload(hl.op.volumes.data(), hl.op.volumes.size(), stream_);
        std::vector<float> fvol(hl.op.volumes.begin(), hl.op.volumes.end());
        d.f.vol.upload(fvol.data(), fvol.size(), stream_);
        d.d.w = hl.weight;
        d.f.w = float(hl.weight);
        d.vol0 = hl.op.volumes.empty() ? 0.0 : hl.op.volumes[0];
        d.const_vol = !hl.op.volumes.empty() && d.vol0 > 0 &&
                      std::all_of(hl.op.volumes.begin(), hl.op.volumes.end(), [&](double v) { return v == d.vol0; });
        d.any_void = std::any_of(hl.op.volumes.begin(), hl.op.volumes.end(), [](double v) { return !(v > 0); });
        if (hl.op.singular) {
            d.ncomp = int(hl.op.comp.volume.size());
            if (d.ncomp > kMaxComponents) throw Error(5, "more ungauged components than the device supports");
            d.comp_volume = hl.op.comp.volume;
            d.slot.upload(hl.op.comp.slot.data(), hl.op.comp.slot.size(), stream_);
        }
        if (l == 0) {
            vol_total_ = 0;
            for (double v : hl.op.volumes)
                if (v > 0) vol_total_ += v;
        }
        if (l + 1 < h.levels.size()) {
            d.nc = int(h.levels[l + 1].op.A.n);
            d.owner.upload(hl.owner.data(), hl.owner.size(), stream_);
            std::vector<int> cptr(static_cast<size_t>(d.nc + 1), 0), ch(hl.owner.size());
            for (int32_t o : hl.owner) cptr[size_t(o + 1)]++;
            for (int J = 0; J < d.nc; ++J) cptr[size_t(J + 1)] += cptr[size_t(J)];
            std::vector<int> nxt(cptr.begin(), cptr.end() - 1);
            for (size_t i = 0; i < hl.owner.size(); ++i) ch[size_t(nxt[size_t(hl.owner[i])]++)] = int(i);
            d.child_ptr.upload(cptr.data(), cptr.size(), stream_);
            d.child.upload(ch.data(), ch.size(), stream_);
            d.d.tinv.upload(hl.transfer_inv.data(), hl.transfer_inv.size(), stream_);
            std::vector<float> ft(hl.transfer_inv.begin(), hl.transfer_inv.end());
            d.f.tinv.upload(ft.data(), ft.size(), stream_);
            d.d.tw = hl.transfer_weight;
            d.f.tw = float(hl.transfer_weight);
        }
        if (l == 0) {
            // open-face conductances of the finest level (true residuals)
            if (std::any_of(hl.op.bdiag.begin(), hl.op.bdiag.end(), [](double v) { return v != 0.0; }))
                bdiag_.upload(hl.op.bdiag.data(), hl.op.bdiag.size(), stream_);
            else
                bdiag_.free();
            open_sides_ = hl.op.any_open();
        }
        if (rb_) {
            std::vector<unsigned char> col = red_black_colours(hl.op.mesh);
            d.rbw = red_black_weight(A, col);
            d.colour.upload(col.data(), col.size(), stream_);
        }
        for (auto* a : {&d.d.x, &d.d.y, &d.d.b, &d.d.r, &d.d.s}) a->alloc(static_cast<size_t>(d.n));
        for (auto* a : {&d.f.x, &d.f.y, &d.f.b, &d.f.r, &d.f.s}) a->alloc(static_cast<size_t>(d.n));
        TPA_CUDA(cudaStreamSynchronize(stream_));  // host staging vectors go out of scope
    }
    coarse_n_ = int(h.coarse_n);
    coarse_inv_.upload(h.coarse_inverse.data(), h.coarse_inverse.size(), stream_);
    coarse_b_.alloc(static_cast<size_t>(coarse_n_));
    coarse_x_.alloc(static_cast<size_t>(coarse_n_));
    const size_t n = size_t(levels_[0].n);
    for (auto* a : {&b_, &r_, &p_, &ap_, &z_, &tmp_}) a->alloc(n);
    TPA_CUDA(cudaStreamSynchronize(stream_));
    build_views();
    upload_structured(h);
    upload_tiles(h);
}

void DeviceSolver::apply(const double* x, double* y) {
    DevLevel& L = levels_[0];
    k_spmv<double><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, L.rowptr.p, L.col.p, L.d.val.p, x, y);
    ++launches_;
    TPA_CUDA(cudaGetLastError());
}

template <typename T>
void DeviceSolver::project_rhs(int l, T* b) {
    DevLevel& L = levels_[size_t(l)];
    for (int s = 0; s < L.ncomp; ++s) {
        const int* slot = L.ncomp > 1 ? L.slot.p : nullptr;
        k_slot_sum<T><<<kReduceBlocks, kThreads, 0, stream_>>>(L.n, b, nullptr, slot, s, 0, partial_.p);
        k_fold_sum<<<1, kThreads, 0, stream_>>>(partial_.p, kReduceBlocks, sums_.p + s);
        k_sub_scaled<T><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, b, lv<T>(l).vol.p, slot, s, sums_.p + s,
                                                                 L.comp_volume[size_t(s)]);
        launches_ += 3;
    }
}

template <typename T>
void DeviceSolver::remove_means(int l, T* x) {
    DevLevel& L = levels_[size_t(l)];
    for (int s = 0; s < L.ncomp; ++s) {
        const int* slot = L.ncomp > 1 ? L.slot.p : nullptr;
        k_slot_sum<T><<<kReduceBlocks, kThreads, 0, stream_>>>(L.n, x, lv<T>(l).vol.p, slot, s, 1, partial_.p);
        k_fold_sum<<<1, kThreads, 0, stream_>>>(partial_.p, kReduceBlocks, sums_.p + s);
        k_sub_scaled<T><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, x, nullptr, slot, s, sums_.p + s,
                                                                 L.comp_volume[size_t(s)]);
        launches_ += 3;
    }
}

// V-cycle on the level vectors of precision T: rhs in lv<T>(0).b, result in lv<T>(0).x.
template <typename T>
void DeviceSolver::vcycle_t(int /*unused*/) {
    const int nl = int(levels_.size());
    std::vector<T*> xcur(static_cast<size_t>(nl));
    for (int l = 0; l < nl - 1; ++l) {
        DevLevel& L = levels_[size_t(l)];
        DevLevelT<T>& D = lv<T>(l);
        if (L.ncomp) project_rhs<T>(l, D.b.p);
        T* x = D.x.p;
        T* y = D.y.p;
        if (rb_) {
            // red then black per sweep, from x = 0
            k_fill<T><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, x, T(0));
            for (int k = 0; k < pre_; ++k)
                for (int c : {0, 1}) {
                    k_rb_sweep<T><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, L.rowptr.p, L.col.p, D.val.p, D.b.p,
                                                                          D.dinv.p, L.colour.p, c, T(L.rbw), x, y);
                    std::swap(x, y);
                }
            launches_ += 1 + pre_;  // with the count below: the fill and 2 pre_ half-sweeps
        } else if (pre_ == 0) {
            k_fill<T><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, x, T(0));
        } else {
            k_jacobi_first<T><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, D.b.p, D.dinv.p, D.w, x);
            for (int k = 1; k < pre_; ++k) {
                k_jacobi<T><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, L.rowptr.p, L.col.p, D.val.p, D.b.p,
                                                                     D.dinv.p, D.w, x, y);
                std::swap(x, y);
            }
        }
        launches_ += pre_ ? pre_ : 1;
        xcur[size_t(l)] = x;
        k_residual<T><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, L.rowptr.p, L.col.p, D.val.p, D.b.p, x, D.tinv.p,
                                                               D.r.p, D.s.p);
        k_restrict<T><<<grid_for(L.nc), kThreads, 0, stream_>>>(L.nc, L.child_ptr.p, L.child.p, L.rowptr.p, L.col.p,
                                                                D.val.p, D.r.p, D.s.p, D.tw, lv<T>(l + 1).b.p);
        launches_ += 2;
    }
    {
        const int l = nl - 1;
        DevLevel& L = levels_[size_t(l)];
        DevLevelT<T>& D = lv<T>(l);
        if (L.ncomp) project_rhs<T>(l, D.b.p);
        double* cb = reinterpret_cast<double*>(D.b.p);
        double* cx = reinterpret_cast<double*>(D.x.p);
        if (sizeof(T) != sizeof(double)) {
            k_convert<T, double><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, D.b.p, coarse_b_.p);
            cb = coarse_b_.p;
            cx = coarse_x_.p;
            ++launches_;
        }
        k_coarse<<<grid_for(int64_t(L.n) * 32), kThreads, 0, stream_>>>(coarse_n_, coarse_inv_.p, cb, cx);
        ++launches_;
        if (sizeof(T) != sizeof(double)) {
            k_convert<double, T><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, coarse_x_.p, D.x.p);
            ++launches_;
        }
        xcur[size_t(l)] = D.x.p;
    }
    for (int l = nl - 2; l >= 0; --l) {
        DevLevel& L = levels_[size_t(l)];
        DevLevelT<T>& D = lv<T>(l);
        T* x = xcur[size_t(l)];
        T* y = (x == D.x.p) ? D.y.p : D.x.p;
        k_prolong<T><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, L.rowptr.p, L.col.p, D.val.p, L.owner.p,
                                                              xcur[size_t(l + 1)], D.tinv.p, D.tw, x);
        ++launches_;
        for (int k = 0; k < post_; ++k) {
            if (rb_) {  // black then red: the reverse of the pre-smoothing
                for (int c : {1, 0}) {
                    k_rb_sweep<T><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, L.rowptr.p, L.col.p, D.val.p, D.b.p,
                                                                          D.dinv.p, L.colour.p, c, T(L.rbw), x, y);
                    std::swap(x, y);
                    ++launches_;
                }
                continue;
            }
            k_jacobi<T><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, L.rowptr.p, L.col.p, D.val.p, D.b.p, D.dinv.p,
                                                                 D.w, x, y);
            std::swap(x, y);
            ++launches_;
        }
        xcur[size_t(l)] = x;
    }
    if (nl == 1) {
        // single level: the coarse solve already produced x
    }
    // result into lv<T>(0).x
    if (xcur[0] != lv<T>(0).x.p)
        TPA_CUDA(cudaMemcpyAsync(lv<T>(0).x.p, xcur[0], sizeof(T) * size_t(levels_[0].n), cudaMemcpyDeviceToDevice,
                                 stream_));
    if (levels_[0].ncomp && nl > 1) remove_means<T>(0, lv<T>(0).x.p);
    TPA_CUDA(cudaGetLastError());
}

void DeviceSolver::vcycle(const double* r, double* z, int precision) {
    const int n = levels_[0].n;
    if (fused_ok_) {
        vcycle_fused(r, z, precision);
        return;
    }
    if (precision == 0) {
        TPA_CUDA(cudaMemcpyAsync(levels_[0].d.b.p, r, sizeof(double) * size_t(n), cudaMemcpyDeviceToDevice, stream_));
        vcycle_t<double>(0);
        TPA_CUDA(cudaMemcpyAsync(z, levels_[0].d.x.p, sizeof(double) * size_t(n), cudaMemcpyDeviceToDevice, stream_));
    } else {
        k_convert<double, float><<<grid_for(n), kThreads, 0, stream_>>>(n, r, levels_[0].f.b.p);
        vcycle_t<float>(0);
        k_convert<float, double><<<grid_for(n), kThreads, 0, stream_>>>(n, levels_[0].f.x.p, z);
        launches_ += 2;
    }
}

double DeviceSolver::time_kernel(int which, int level, int precision, int iters) {
    if (fused_ok_) return time_fused(which, level, precision, iters);
    if (level < 0 || level >= int(levels_.size())) throw Error(1, "bad level");
    if (which != 3 && level == int(levels_.size()) - 1) throw Error(1, "the coarsest level has no such kernel");
    if (which == 3 && level != 0) throw Error(1, "the CG operator lives on the finest level");
    DevLevel& L = levels_[size_t(level)];
    cudaEvent_t e0, e1;
    TPA_CUDA(cudaEventCreate(&e0));
    TPA_CUDA(cudaEventCreate(&e1));
    auto launch = [&]() {
        if (precision == 0) {
            DevLevelT<double>& D = L.d;
            if (which == 0)
                k_jacobi<double><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, L.rowptr.p, L.col.p, D.val.p, D.b.p,
                                                                          D.dinv.p, D.w, D.x.p, D.y.p);
            else if (which == 1) {
                k_residual<double><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, L.rowptr.p, L.col.p, D.val.p, D.b.p,
                                                                            D.x.p, D.tinv.p, D.r.p, D.s.p);
                k_restrict<double><<<grid_for(L.nc), kThreads, 0, stream_>>>(L.nc, L.child_ptr.p, L.child.p, L.rowptr.p,
                                                                             L.col.p, D.val.p, D.r.p, D.s.p, D.tw,
                                                                             lv<double>(level + 1).b.p);
            } else if (which == 2)
                k_prolong<double><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, L.rowptr.p, L.col.p, D.val.p,
                                                                           L.owner.p, lv<double>(level + 1).x.p,
                                                                           D.tinv.p, D.tw, D.x.p);
            else
                k_cg_ap<<<kReduceBlocks, kThreads, 0, stream_>>>(L.n, L.rowptr.p, L.col.p, D.val.p, D.x.p, D.y.p,
                                                                   partial_.p);
        } else {
            DevLevelT<float>& D = L.f;
            if (which == 0)
                k_jacobi<float><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, L.rowptr.p, L.col.p, D.val.p, D.b.p,
                                                                         D.dinv.p, D.w, D.x.p, D.y.p);
            else if (which == 1) {
                k_residual<float><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, L.rowptr.p, L.col.p, D.val.p, D.b.p,
                                                                           D.x.p, D.tinv.p, D.r.p, D.s.p);
                k_restrict<float><<<grid_for(L.nc), kThreads, 0, stream_>>>(L.nc, L.child_ptr.p, L.child.p, L.rowptr.p,
                                                                            L.col.p, D.val.p, D.r.p, D.s.p, D.tw,
                                                                            lv<float>(level + 1).b.p);
            } else if (which == 2)
                k_prolong<float><<<grid_for(L.n), kThreads, 0, stream_>>>(L.n, L.rowptr.p, L.col.p, D.val.p,
                                                                          L.owner.p, lv<float>(level + 1).x.p,
                                                                          D.tinv.p, D.tw, D.x.p);
            else
                throw Error(1, "the CG operator runs in FP64 only");
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

void DeviceSolver::residual_norms(const double* r, double out[2]) {
    DevLevel& L = levels_[0];
    const double* vol = L.d.vol.p;
    k_l2_terms<<<kReduceBlocks, kThreads, 0, stream_>>>(L.n, r, vol, partial_.p);
    k_fold_sum<<<1, kThreads, 0, stream_>>>(partial_.p, kReduceBlocks, sums_.p + 56);
    k_fold_sum<<<1, kThreads, 0, stream_>>>(partial_.p + kReduceBlocks, kReduceBlocks, sums_.p + 57);
    launches_ += 3;
    strong_max(r, sums_.p + 58);
    TPA_CUDA(cudaMemcpyAsync(host_d_, sums_.p + 56, 3 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    TPA_CUDA(cudaStreamSynchronize(stream_));
    out[0] = std::sqrt(host_d_[0] / host_d_[1]);
    out[1] = host_d_[2];
}

double DeviceSolver::read_scalar(const double* dev) {
    TPA_CUDA(cudaMemcpyAsync(host_d_, dev, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    TPA_CUDA(cudaStreamSynchronize(stream_));
    return host_d_[0];
}

void DeviceSolver::strong_max(const double* r, double* out) {
    DevLevel& L = levels_[0];
    k_strong_max<<<kReduceBlocks, kThreads, 0, stream_>>>(L.n, r, L.d.vol.p, partial_.p);
    k_fold_max<<<1, kThreads, 0, stream_>>>(partial_.p, kReduceBlocks, out);
    launches_ += 2;
}

void DeviceSolver::solve(const double* rhs, double* x_user, double rtol, double atol, int max_cycles,
                         int compatibility, int precision, SolveStats& st) {
    // The solve works on an internal copy of the iterate so that the captured
    // CG graph always sees the same addresses.
    double* x = xw_.p;
    TPA_CUDA(cudaSetDevice(device_));
    if (!(rtol >= 0 && rtol < 1)) throw Error(1, "rtol must lie in [0, 1)");
    if (!(atol >= 0)) throw Error(1, "atol must be nonnegative");
    if (max_cycles < 0) throw Error(1, "max_cycles must be nonnegative");
    if (compatibility != 0 && compatibility != 1) throw Error(1, "compatibility must be :project or :error");
    if (precision < 0 || precision > 2)
        throw Error(1, "precision must be 0 (FP64), 1 (mixed) or 2 (mixed with FP32 Krylov vectors)");
    if (precision == 2 && (!fused_ok_ || std::getenv("TPAGMG_PLAIN_SOLVE")))
        throw Error(5, "the refinement solve needs the fused cycle (two pre- and two post-sweeps, one component)");
    if (fused_ok_ && !std::getenv("TPAGMG_PLAIN_SOLVE")) {
        solve_fast(rhs, x_user, rtol, atol, max_cycles, compatibility, precision, st);
        return;
    }
    const double eps = 2.220446049250313e-16;
    DevLevel& L = levels_[0];
    const int n = L.n;
    const double* vol = L.d.vol.p;
    const int g = grid_for(n);
    cudaEvent_t e0, e1;
    TPA_CUDA(cudaEventCreate(&e0));
    TPA_CUDA(cudaEventCreate(&e1));
    TPA_CUDA(cudaEventRecord(e0, stream_));
    st = SolveStats();
    TPA_CUDA(cudaMemcpyAsync(x, x_user, sizeof(double) * size_t(n), cudaMemcpyDeviceToDevice, stream_));
    k_scale_rhs<<<g, kThreads, 0, stream_>>>(n, rhs, vol, b_.p, x);
    ++launches_;
    double removed = 0;
    if (L.ncomp) {
        double total = 0, tvol = 0;
        for (int s = 0; s < L.ncomp; ++s) {
            const int* slot = L.ncomp > 1 ? L.slot.p : nullptr;
            k_slot_sum<double><<<kReduceBlocks, kThreads, 0, stream_>>>(n, b_.p, nullptr, slot, s, 0, partial_.p);
            k_fold_sum<<<1, kThreads, 0, stream_>>>(partial_.p, kReduceBlocks, sums_.p + s);
            k_slot_sum<double><<<kReduceBlocks, kThreads, 0, stream_>>>(n, b_.p, nullptr, slot, s, 2, partial_.p);
            k_fold_sum<<<1, kThreads, 0, stream_>>>(partial_.p, kReduceBlocks, sums_.p + 32 + s);
            launches_ += 4;
            TPA_CUDA(cudaMemcpyAsync(host_d_, sums_.p + s, sizeof(double), cudaMemcpyDeviceToHost, stream_));
            TPA_CUDA(cudaMemcpyAsync(host_d_ + 1, sums_.p + 32 + s, sizeof(double), cudaMemcpyDeviceToHost, stream_));
            TPA_CUDA(cudaStreamSynchronize(stream_));
            double ssum = host_d_[0], sabs = host_d_[1];
            if (compatibility == 1 && std::fabs(ssum) > 256 * eps * std::max(1.0, sabs))
                throw Error(1, "Poisson right-hand side has nonzero volume mean");
            total += ssum;
            tvol += L.comp_volume[size_t(s)];
            const double cm = std::fabs(ssum / L.comp_volume[size_t(s)]);
            if (!std::isfinite(cm) || cm > st.removed_max_component_mean) st.removed_max_component_mean = cm;
            k_sub_scaled<double><<<g, kThreads, 0, stream_>>>(n, b_.p, vol, slot, s, sums_.p + s,
                                                              L.comp_volume[size_t(s)]);
            ++launches_;
        }
        removed = tvol ? total / tvol : 0;
        remove_means<double>(0, x);
    }
    auto residual = [&](const double* xx, double* rr) {
        k_residual64<<<g, kThreads, 0, stream_>>>(n, L.rowptr.p, L.col.p, L.d.val.p, b_.p, xx, rr, bdiag_.p);
        ++launches_;
    };
    auto norms = [&](const double* rr, double& l2, double& linf) {
        k_l2_terms<<<kReduceBlocks, kThreads, 0, stream_>>>(n, rr, vol, partial_.p);
        k_fold_sum<<<1, kThreads, 0, stream_>>>(partial_.p, kReduceBlocks, sums_.p + 48);
        k_fold_sum<<<1, kThreads, 0, stream_>>>(partial_.p + kReduceBlocks, kReduceBlocks, sums_.p + 49);
        strong_max(rr, sums_.p + 50);
        launches_ += 3;
        TPA_CUDA(cudaMemcpyAsync(host_d_, sums_.p + 48, 3 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        TPA_CUDA(cudaStreamSynchronize(stream_));
        l2 = std::sqrt(host_d_[0] / host_d_[1]);
        linf = host_d_[2];
    };
    auto floor_of = [&](const double* xx) {
        // 128 eps max(1, max(|A||x| / V, |b| / V)) on the assembled |A|
        k_abs_spmv<<<g, kThreads, 0, stream_>>>(n, L.rowptr.p, L.col.p, L.d.val.p, xx, tmp_.p);
        ++launches_;
        strong_max(tmp_.p, sums_.p + 51);
        strong_max(b_.p, sums_.p + 52);
        TPA_CUDA(cudaMemcpyAsync(host_d_, sums_.p + 51, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        TPA_CUDA(cudaStreamSynchronize(stream_));
        return 128 * eps * std::max(1.0, std::max(host_d_[0], host_d_[1]));
    };
    auto guarded = [&](const double* xx, double target, double init, double cur) {
        if (!(std::isfinite(init) && std::isfinite(cur) && target < cur && cur < init)) return target;
        double fl = floor_of(xx);
        return (std::isfinite(fl) && fl < init / 100) ? std::max(target, fl) : target;
    };
    residual(x, r_.p);
    double init_l2, init_linf;
    norms(r_.p, init_l2, init_linf);
    double floor = floor_of(x);
    double target = std::max(atol, std::max(rtol * std::max(init_linf, eps), floor));
    int total = 0;
    if (init_linf > target) {
        while (total < max_cycles && fused_ok_) {
            int niter = 0, flags = 0;
            cg_fused(precision, target, max_cycles - total, niter, flags);
            total += niter;
            if (L.ncomp) remove_means<double>(0, x);
            residual(x, r_.p);
            strong_max(r_.p, sums_.p + 53);
            double final_linf = read_scalar(sums_.p + 53);
            double eff = guarded(x, target, init_linf, final_linf);
            ++st.restarts;
            if (final_linf <= eff) break;
            if (!std::isfinite(final_linf) || niter == 0) break;
        }
        while (total < max_cycles && !fused_ok_) {
            // Krylov.jl cg! warm-started at x: r = b - A x, z = M r, p = z, gamma = r'z
            residual(x, r_.p);
            vcycle(r_.p, z_.p, precision);
            TPA_CUDA(cudaMemcpyAsync(p_.p, z_.p, sizeof(double) * size_t(n), cudaMemcpyDeviceToDevice, stream_));
            k_dot<<<kReduceBlocks, kThreads, 0, stream_>>>(n, r_.p, z_.p, partial_.p);
            k_cg_init<<<1, kThreads, 0, stream_>>>(partial_.p, kReduceBlocks, sc_.p, target);
            launches_ += 2;
            int niter = 0;
            const int itmax = max_cycles - total;
            TPA_CUDA(cudaMemcpyAsync(host_sc_, sc_.p, sizeof(CgScalars), cudaMemcpyDeviceToHost, stream_));
            TPA_CUDA(cudaStreamSynchronize(stream_));
            bool stop = (host_sc_->flags & 8) || itmax <= 0;
            while (!stop) {
                k_cg_ap<<<kReduceBlocks, kThreads, 0, stream_>>>(n, L.rowptr.p, L.col.p, L.d.val.p, p_.p, ap_.p,
                                                                   partial_.p);
                k_cg_alpha<<<1, kThreads, 0, stream_>>>(partial_.p, kReduceBlocks, sc_.p);
                k_cg_update<<<kReduceBlocks, kThreads, 0, stream_>>>(n, x, r_.p, p_.p, ap_.p, vol, sc_.p,
                                                                       partial_.p + kReduceBlocks);
                launches_ += 3;
                vcycle(r_.p, z_.p, precision);
                k_dot<<<kReduceBlocks, kThreads, 0, stream_>>>(n, r_.p, z_.p, partial_.p);
                k_cg_beta<<<1, kThreads, 0, stream_>>>(partial_.p, kReduceBlocks, sc_.p);
                k_cg_p<<<g, kThreads, 0, stream_>>>(n, p_.p, z_.p, sc_.p);
                launches_ += 3;
                TPA_CUDA(cudaMemcpyAsync(host_sc_, sc_.p, sizeof(CgScalars), cudaMemcpyDeviceToHost, stream_));
                TPA_CUDA(cudaStreamSynchronize(stream_));
                niter = host_sc_->iter;
                stop = (host_sc_->flags & 7) || niter >= itmax;
            }
            total += niter;
            if (L.ncomp) remove_means<double>(0, x);
            residual(x, r_.p);
            strong_max(r_.p, sums_.p + 53);
            double final_linf = read_scalar(sums_.p + 53);
            double eff = guarded(x, target, init_linf, final_linf);
            ++st.restarts;
            if (final_linf <= eff) break;
            if (!std::isfinite(final_linf) || niter == 0) break;
        }
    }
    if (L.ncomp) remove_means<double>(0, x);
    residual(x, r_.p);
    double fin_l2, fin_linf;
    norms(r_.p, fin_l2, fin_linf);
    target = guarded(x, target, init_linf, fin_linf);
    TPA_CUDA(cudaMemcpyAsync(x_user, x, sizeof(double) * size_t(n), cudaMemcpyDeviceToDevice, stream_));
    TPA_CUDA(cudaEventRecord(e1, stream_));
    TPA_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    st.cycles = total;
    st.converged = std::isfinite(fin_linf) && std::isfinite(target) && fin_linf <= target;
    st.initial_l2 = init_l2;
    st.initial_linf = init_linf;
    st.final_l2 = fin_l2;
    st.final_linf = fin_linf;
    st.target_linf = target;
    st.residual_scale = std::max(init_linf, eps);
    st.removed_rhs_mean = removed;
    st.ms_total = ms;
}

}  // namespace tpa
