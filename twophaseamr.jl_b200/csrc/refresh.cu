// Device-side coefficient refresh: `_refresh_geometric_multigrid!`
// (src/solvers/multigrid/geometric_preconditioner.jl:483-594 of
// ronaldremmerswaal/TwoPhaseAMR.jl) on the uploaded topology.  New finest-level
// face coefficients kappa are restricted level by level (tree_coarsening.jl:
// 538-555), every level operator S = J' sqrt(k) K sqrt(k) J (elliptic.jl:
// 175-257, 847-916) is re-evaluated on its fixed sparsity pattern, the Jacobi
// and transfer weights are recomputed (hierarchy.jl:8-30, 631-721), and the
// augmented coarsest matrix is factored again (geometric_preconditioner.jl:
// 6-24, 144-169) -- all on the GPU.
//
// The pattern of S and the contributions to each entry depend on the topology
// only, so they are listed once on the host: entry k of the symmetric operator
// is sum_t c_t * sqrt(kappa_f) * sqrt(kappa_g) (kappa_f when f = g) over its
// terms t, each raw contribution split half to (r, c) and half to (c, r) as in
// the symmetric average (A + A')/2.  Sums run in a fixed order (deterministic).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include <cooperative_groups.h>

#include "device.cuh"

namespace tpa {
namespace {

constexpr int kRThreads = 256;

int rgrid(int64_t n) {
    int64_t g = (n + kRThreads - 1) / kRThreads;
    return int(std::max<int64_t>(1, std::min<int64_t>(g, 1184)));
}

__global__ void kr_sqrt(int n, const double* __restrict__ k, double* __restrict__ sk) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) sk[i] = sqrt(k[i]);
}

// coarse face coefficients: overlap-weighted average of the fine ones
__global__ void kr_restrict(int nfc, const int* __restrict__ rptr, const int* __restrict__ ridx,
                            const double* __restrict__ rw, const double* __restrict__ kf, double* __restrict__ kc) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nfc; f += gridDim.x * blockDim.x) {
        double v = 0.0;
        for (int k = rptr[f]; k < rptr[f + 1]; ++k) v += rw[k] * kf[ridx[k]];
        kc[f] = v;
    }
}

// entries of the symmetric operator from their listed terms
__global__ void kr_assemble(int nnz, const int* __restrict__ tptr, const int* __restrict__ tf,
                            const int* __restrict__ tg, const double* __restrict__ tc,
                            const double* __restrict__ kappa, const double* __restrict__ sk, double* __restrict__ vd,
                            float* __restrict__ vf) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x) {
        double v = 0.0;
        for (int t = tptr[k]; t < tptr[k + 1]; ++t) {
            const int f = tf[t], g = tg[t];
            v += tc[t] * (f == g ? kappa[f] : sk[f] * sk[g]);
        }
        if (v == 0.0) v = 0.0;  // no negative zeros
        vd[k] = v;
        vf[k] = float(v);
    }
}

// D^-1 and Dt^-1 per row and the two Jacobi bounds max_i sum_j |a_ij| / a_ii;
// the last block writes w = min(1, 4/(3 bound)) (1 without a bound) and the
// unclamped transfer weight 4/(3 bound) (0 without a bound) into wtw[0..1].
__global__ void kr_weights(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ val, int singular, double* __restrict__ dinv_d,
                           float* __restrict__ dinv_f, double* __restrict__ tinv_d, float* __restrict__ tinv_f,
                           double* partial, unsigned* counter, double* wtw, int* err) {
    double bs = 0.0, bt = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = 0.0, rs = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            rs += fabs(val[k]);
            if (ci[k] == i) d = val[k];
        }
        double di = d;
        if (d == 0.0 && singular) {
            // an isolated cell of an ungauged component keeps D^-1 = 0
        } else if (!(d > 0)) {
            atomicExch(err, 1);
        } else {
            bs = fmax(bs, rs / d);
            di = 1.0 / d;
        }
        dinv_d[i] = di;
        dinv_f[i] = float(di);
        if (tinv_d) {
            double ti = d;
            if (d > 0) {
                bt = fmax(bt, rs / d);
                ti = 1.0 / d;
            }
            tinv_d[i] = ti;
            tinv_f[i] = float(ti);
        }
    }
    __shared__ double sh[2][32];
    __shared__ bool last;
    for (int o = 16; o; o >>= 1) {
        bs = fmax(bs, __shfl_down_sync(0xffffffffu, bs, o));
        bt = fmax(bt, __shfl_down_sync(0xffffffffu, bt, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (!lane) {
        sh[0][wid] = bs;
        sh[1][wid] = bt;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ms = 0.0, mt = 0.0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) {
            ms = fmax(ms, sh[0][w]);
            mt = fmax(mt, sh[1][w]);
        }
        partial[blockIdx.x] = ms;
        partial[gridDim.x + blockIdx.x] = mt;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double ms = 0.0, mt = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) {
            ms = fmax(ms, ((volatile double*)partial)[b]);
            mt = fmax(mt, ((volatile double*)partial)[gridDim.x + b]);
        }
        wtw[0] = ms == 0.0 ? 1.0 : fmin(1.0, 4.0 / (3.0 * ms));
        wtw[1] = mt == 0.0 ? 0.0 : 4.0 / (3.0 * mt);
        *counter = 0;
    }
}

// the augmented coarsest matrix [A v; v' 0] (M zeroed before)
__global__ void kr_coarse_fill(int n, int N, const int* __restrict__ rp, const int* __restrict__ ci,
                               const double* __restrict__ val, const int* __restrict__ slot,
                               const double* __restrict__ vol, int ncomp, double* __restrict__ M) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        for (int k = rp[r]; k < rp[r + 1]; ++k) M[size_t(r) * N + ci[k]] = val[k];
        if (ncomp) {
            const int s = slot ? slot[r] : 0;
            if (s >= 0) {
                M[size_t(r) * N + n + s] = vol[r];
                M[size_t(n + s) * N + r] = vol[r];
            }
        }
    }
}

// (value, row) pairs: the larger value wins, ties go to the smaller row (the
// first maximum of a sequential scan)
__device__ __forceinline__ void better(double& v, int& i, double ov, int oi) {
    if (ov > v || (ov == v && oi < i)) {
        v = ov;
        i = oi;
    }
}

template <bool Cl>
__device__ __forceinline__ void lu_sync() {
    if constexpr (Cl) cooperative_groups::this_cluster().sync();
    else __syncthreads();
}

// LU with partial pivoting of the augmented coarsest matrix M (N x N,
// row-major, overwritten by the factors; piv[k] = row exchanged with row k).
// Cl: the rows are spread cyclically over the CTAs of a thread-block cluster
// (row r on CTA r % C at local row r / C) and held in shared memory, each CTA
// reading the pivot row and the candidates of the others through distributed
// shared memory; otherwise one CTA works on M in global memory.  Each step
// follows the host factorisation operation for operation: the pivot is the
// first row of largest |M[r][k]| (r >= k), rows k and p are exchanged whole,
// l = M[r][k] * (1 / M[k][k]) overwrites M[r][k] and M[r][c] -= l M[k][c]
// (c > k, l != 0).  The search for the next pivot is fused into the update.
// err = 2 on a zero pivot.
template <bool Cl>
__global__ void __launch_bounds__(1024) kr_lu(int N, double* __restrict__ M, int* __restrict__ piv, int* err) {
    namespace cg = cooperative_groups;
    extern __shared__ double lu_sm[];
    __shared__ double wv[32];
    __shared__ int wi[32];
    __shared__ double cand_v;
    __shared__ int cand_i;
    __shared__ int pivot;
    int C = 1, rank = 0;
    if constexpr (Cl) {
        C = int(cg::this_cluster().num_blocks());
        rank = int(cg::this_cluster().block_rank());
    }
    const int R = (N + C - 1) / C;
    double* rows = Cl ? lu_sm : M;
    double* prow = Cl ? lu_sm + size_t(R) * N : lu_sm;
    double* trow = prow + N;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = int(blockDim.x >> 5);
    auto first_local = [&](int j) {  // smallest local row whose global row is >= j
        const int t = j - rank;
        return t <= 0 ? 0 : (t + C - 1) / C;
    };
    auto row_of = [&](int owner, int r) -> double* {
        double* base = rows;
        if constexpr (Cl) base = cg::this_cluster().map_shared_rank(rows, owner);
        return base + size_t(r / C) * N;
    };
    auto publish = [&](double bv, int bi) {  // this CTA's candidate into cand_v / cand_i
        for (int o = 16; o; o >>= 1) better(bv, bi, __shfl_down_sync(0xffffffffu, bv, o),
                                            __shfl_down_sync(0xffffffffu, bi, o));
        if (!lane) {
            wv[wid] = bv;
            wi[wid] = bi;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double v = wv[0];
            int i = wi[0];
            for (int w = 1; w < nw; ++w) better(v, i, wv[w], wi[w]);
            cand_v = v;
            cand_i = i;
        }
    };
    if constexpr (Cl) {
        for (int lr = 0; lr < R && lr * C + rank < N; ++lr)
            for (int c = threadIdx.x; c < N; c += blockDim.x)
                rows[size_t(lr) * N + c] = M[size_t(lr * C + rank) * N + c];
        __syncthreads();
    }
    {
        double bv = -1.0;
        int bi = N;
        for (int lr = first_local(0) + int(threadIdx.x); lr < R && lr * C + rank < N; lr += blockDim.x)
            better(bv, bi, fabs(rows[size_t(lr) * N]), lr * C + rank);
        publish(bv, bi);
    }
    lu_sync<Cl>();
    for (int k = 0; k < N; ++k) {
        if (wid == 0) {
            double v = -1.0;
            int i = N;
            if (lane < C) {
                if constexpr (Cl) {
                    v = *cg::this_cluster().map_shared_rank(&cand_v, lane);
                    i = *cg::this_cluster().map_shared_rank(&cand_i, lane);
                } else {
                    v = cand_v;
                    i = cand_i;
                }
            }
            for (int o = 16; o; o >>= 1) better(v, i, __shfl_down_sync(0xffffffffu, v, o),
                                                __shfl_down_sync(0xffffffffu, i, o));
            if (lane == 0) {
                pivot = (v > 0.0 && i < N) ? i : -1;
                if (rank == 0) piv[k] = i < N ? i : k;
            }
        }
        __syncthreads();
        const int p = pivot;
        if (p < 0) {
            if (rank == 0 && threadIdx.x == 0) atomicExch(err, 2);
            break;  // every CTA takes the same decision
        }
        const double* src_p = row_of(p % C, p);
        for (int c = threadIdx.x; c < N; c += blockDim.x) prow[c] = src_p[c];
        if (p != k && rank == p % C) {
            const double* src_k = row_of(k % C, k);
            for (int c = threadIdx.x; c < N; c += blockDim.x) trow[c] = src_k[c];
        }
        lu_sync<Cl>();  // rows k and p are read everywhere before they change
        if (p != k) {
            if (rank == k % C)
                for (int c = threadIdx.x; c < N; c += blockDim.x) rows[size_t(k / C) * N + c] = prow[c];
            if (rank == p % C)
                for (int c = threadIdx.x; c < N; c += blockDim.x) rows[size_t(p / C) * N + c] = trow[c];
        }
        __syncthreads();
        const double inv = 1.0 / prow[k];
        double bv = -1.0;
        int bi = N;
        for (int lr = first_local(k + 1) + wid; lr < R && lr * C + rank < N; lr += nw) {
            double* row = rows + size_t(lr) * N;
            const double l = row[k] * inv;
            if (l != 0.0)
                for (int c = k + 1 + lane; c < N; c += 32) row[c] -= l * prow[c];
            __syncwarp();
            if (lane == 0) {
                row[k] = l;
                if (k + 1 < N) better(bv, bi, fabs(row[k + 1]), lr * C + rank);
            }
        }
        publish(bv, bi);
        lu_sync<Cl>();  // updates and candidates complete before the next step
    }
    lu_sync<Cl>();  // no CTA leaves while another may still read its rows
    if constexpr (Cl) {
        for (int lr = 0; lr < R && lr * C + rank < N; ++lr)
            for (int c = threadIdx.x; c < N; c += blockDim.x)
                M[size_t(lr * C + rank) * N + c] = rows[size_t(lr) * N + c];
    }
}

// The first n columns of M^-1 from the factors, one warp per column: e = P
// e_col (a unit vector: only its position moves), forward substitution with
// the unit lower factor (rows above the 1 stay zero), back substitution with
// the upper factor; G[r][col] = e[r] for r < n.  Dot products run across the
// lanes with a fixed shuffle tree (deterministic).
__global__ void __launch_bounds__(128) kr_coarse_inv(int N, int n, const double* __restrict__ M,
                                                     const int* __restrict__ piv, double* __restrict__ G,
                                                     const int* __restrict__ err) {
    extern __shared__ double inv_sm[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int col = int(blockIdx.x) * int(blockDim.x >> 5) + wid;
    if (col >= n || *err) return;  // whole warps; no block-wide barrier follows
    double* e = inv_sm + size_t(wid) * N;
    int pos = col;
    for (int k = 0; k < N; ++k) {
        const int p = piv[k];
        if (pos == k) pos = p;
        else if (pos == p) pos = k;
    }
    for (int r = lane; r < N; r += 32) e[r] = r == pos ? 1.0 : 0.0;
    __syncwarp();
    for (int r = pos + 1; r < N; ++r) {
        const double* Mr = M + size_t(r) * N;
        double s = 0.0;
        for (int k = pos + lane; k < r; k += 32) s += Mr[k] * e[k];
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) e[r] -= s;
        __syncwarp();
    }
    for (int r = N - 1; r >= 0; --r) {
        const double* Mr = M + size_t(r) * N;
        double s = 0.0;
        for (int k = r + 1 + lane; k < N; k += 32) s += Mr[k] * e[k];
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) e[r] = (e[r] - s) / Mr[r];
        __syncwarp();
    }
    for (int r = lane; r < n; r += 32) G[size_t(r) * n + col] = e[r];
}

constexpr int kLuCluster = 8;      // CTAs sharing the rows of the coarsest matrix
constexpr int kLuClusterThreads = 512;
constexpr int kInvWarps = 4;       // columns of the inverse per CTA

}  // namespace

// Terms of every operator entry and the face restrictions, from the host
// hierarchy (topology only; run once per upload).
void DeviceSolver::prepare_refresh(const Hierarchy& h) {
    const int nl = int(h.levels.size());
    rl_.clear();
    rl_.resize(size_t(nl));
    for (int l = 0; l < nl; ++l) {
        const LevelOperator& op = h.levels[size_t(l)].op;
        const Mesh& m = op.mesh;
        const Metric& K = op.metric;
        const Csr& A = op.A;
        const int64_t nf = m.nfaces();
        auto pos = [&](int32_t r, int32_t c) -> int64_t {
            auto b = A.col.begin() + A.ptr[size_t(r)], e = A.col.begin() + A.ptr[size_t(r + 1)];
            auto it = std::lower_bound(b, e, c);
            if (it == e || *it != c) throw Error(7, "operator pattern lacks an entry of the refresh");
            return int64_t(it - A.col.begin());
        };
        // every raw contribution (r, c) of S: coefficient and its face pair
        struct Raw {
            int32_t r, c, f, g;
            double coef;
        };
        std::vector<Raw> raw;
        raw.reserve(size_t(4 * nf + 4 * K.off_val.size()));
        for (int64_t f = 0; f < nf; ++f) {
            const double a = m.farea[size_t(f)], kf = K.diag[size_t(f)];
            const int32_t cm = m.fm[size_t(f)], cp = m.fp[size_t(f)];
            const int32_t ff = int32_t(f);
            raw.push_back({cm, cm, ff, ff, (-a * kf) * -a});
            raw.push_back({cm, cp, ff, ff, (-a * kf) * a});
            raw.push_back({cp, cm, ff, ff, (a * kf) * -a});
            raw.push_back({cp, cp, ff, ff, (a * kf) * a});
        }
        for (size_t k = 0; k < K.off_val.size(); ++k) {
            const int32_t fl = K.off_row[k], fr = K.off_col[k];
            const double al = m.farea[size_t(fl)], ar = m.farea[size_t(fr)];
            const int32_t lc[2] = {m.fm[size_t(fl)], m.fp[size_t(fl)]}, rc[2] = {m.fm[size_t(fr)], m.fp[size_t(fr)]};
            const double ls[2] = {-al, al}, rs[2] = {-ar, ar};
            for (int u = 0; u < 2; ++u)
                for (int v = 0; v < 2; ++v) raw.push_back({lc[u], rc[v], fl, fr, (ls[u] * K.off_val[k]) * rs[v]});
        }
        const int64_t nnz = A.ptr.back();
        std::vector<int64_t> cnt(size_t(nnz) + 1, 0);
        std::vector<int64_t> p1(raw.size()), p2(raw.size());
        for (size_t t = 0; t < raw.size(); ++t) {
            p1[t] = pos(raw[t].r, raw[t].c);
            p2[t] = pos(raw[t].c, raw[t].r);
            ++cnt[size_t(p1[t]) + 1];
            ++cnt[size_t(p2[t]) + 1];
        }
        for (int64_t k = 0; k < nnz; ++k) cnt[size_t(k) + 1] += cnt[size_t(k)];
        const int64_t nterms = cnt[size_t(nnz)];
        if (nterms >= (int64_t(1) << 31)) throw Error(5, "too many operator terms for the device refresh");
        std::vector<int> tptr(cnt.begin(), cnt.end()), tf(static_cast<size_t>(nterms)),
            tg(static_cast<size_t>(nterms));
        std::vector<double> tc(static_cast<size_t>(nterms));
        std::vector<int64_t> nxt(cnt.begin(), cnt.end() - 1);
        for (size_t t = 0; t < raw.size(); ++t)
            for (int64_t q : {p1[t], p2[t]}) {
                const int64_t at = nxt[size_t(q)]++;
                tf[size_t(at)] = raw[t].f;
                tg[size_t(at)] = raw[t].g;
                tc[size_t(at)] = raw[t].coef / 2;
            }
        RefreshLevel& R = rl_[size_t(l)];
        R.nf = int(nf);
        R.nnz = int(nnz);
        R.tptr.upload(tptr.data(), tptr.size(), stream_);
        R.tf.upload(tf.data(), tf.size(), stream_);
        R.tg.upload(tg.data(), tg.size(), stream_);
        R.tc.upload(tc.data(), tc.size(), stream_);
        R.kappa.alloc(size_t(std::max<int64_t>(nf, 1)));
        R.sk.alloc(size_t(std::max<int64_t>(nf, 1)));
        const HostLevel& hl = h.levels[size_t(l)];
        if (l + 1 < nl) {
            std::vector<int> rptr(hl.rptr.begin(), hl.rptr.end());
            R.rptr.upload(rptr.data(), rptr.size(), stream_);
            R.ridx.upload(hl.ridx.data(), hl.ridx.size(), stream_);
            R.rw.upload(hl.rw.data(), hl.rw.size(), stream_);
        }
        TPA_CUDA(cudaStreamSynchronize(stream_));
    }
    const HostLevel& c = h.levels.back();
    const int64_t ncomp = c.op.singular ? int64_t(c.op.comp.volume.size()) : 0;
    coarse_N_ = int(c.op.A.n + ncomp);
    coarse_ncomp_ = int(ncomp);
    coarse_M_.alloc(size_t(coarse_N_) * size_t(coarse_N_));
    {
        // the cluster LU when a cluster's shared memory holds the matrix
        const int N = coarse_N_;
        const size_t cl_bytes = (size_t((N + kLuCluster - 1) / kLuCluster) * N + 2 * size_t(N)) * sizeof(double);
        int optin = 0;
        TPA_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_));
        lu_cluster_ = cl_bytes + 1024 <= size_t(optin) && !std::getenv("TPAGMG_LU_ONE_CTA");
        if (lu_cluster_) {
            TPA_CUDA(cudaFuncSetAttribute(kr_lu<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(cl_bytes)));
            cudaLaunchConfig_t cfg;
            std::memset(&cfg, 0, sizeof(cfg));
            cfg.gridDim = dim3(kLuCluster);
            cfg.blockDim = dim3(kLuClusterThreads);
            cfg.dynamicSmemBytes = cl_bytes;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = kLuCluster;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, kr_lu<true>, &cfg) != cudaSuccess || clusters < 1) {
                cudaGetLastError();
                lu_cluster_ = false;
            }
        }
        const size_t inv_bytes = size_t(kInvWarps) * size_t(N) * sizeof(double);
        TPA_CUDA(cudaFuncSetAttribute(kr_coarse_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, int(inv_bytes)));
    }
    coarse_piv_.alloc(size_t(coarse_N_));
    rwtw_.alloc(size_t(2 * nl));
    rpart_.alloc(size_t(2 * 1184));
    rcnt_.alloc(1);
    rerr_.alloc(1);
    TPA_CUDA(cudaMemsetAsync(rcnt_.p, 0, sizeof(unsigned), stream_));
    TPA_CUDA(cudaMemsetAsync(coarse_piv_.p, 0, sizeof(int) * coarse_piv_.n, stream_));
    TPA_CUDA(cudaStreamSynchronize(stream_));
    rl_ready_ = true;
}

bool DeviceSolver::refresh_applicable(const Hierarchy& h) const {
    if (structured_levels() > 0) return false;  // stencil copies hold coefficients of their own
    const HostLevel& c = h.levels.back();
    const int64_t N = c.op.A.n + (c.op.singular ? int64_t(c.op.comp.volume.size()) : 0);
    return N <= kRefreshMaxCoarse;
}

void DeviceSolver::refresh_on_device(const Hierarchy& h, const double* kappa_host) {
    TPA_CUDA(cudaSetDevice(device_));
    if (!rl_ready_) prepare_refresh(h);
    const int nl = int(levels_.size());
    cudaStream_t s = stream_;
    TPA_CUDA(cudaMemsetAsync(rerr_.p, 0, sizeof(int), s));
    TPA_CUDA(cudaMemcpyAsync(rl_[0].kappa.p, kappa_host, sizeof(double) * size_t(rl_[0].nf), cudaMemcpyHostToDevice,
                             s));
    for (int l = 0; l < nl; ++l) {
        RefreshLevel& R = rl_[size_t(l)];
        DevLevel& L = levels_[size_t(l)];
        if (R.nf > 0) kr_sqrt<<<rgrid(R.nf), kRThreads, 0, s>>>(R.nf, R.kappa.p, R.sk.p);
        kr_assemble<<<rgrid(R.nnz), kRThreads, 0, s>>>(R.nnz, R.tptr.p, R.tf.p, R.tg.p, R.tc.p, R.kappa.p, R.sk.p,
                                                      L.d.val.p, L.f.val.p);
        if (l + 1 < nl && rl_[size_t(l + 1)].nf > 0)
            kr_restrict<<<rgrid(rl_[size_t(l + 1)].nf), kRThreads, 0, s>>>(rl_[size_t(l + 1)].nf, R.rptr.p, R.ridx.p,
                                                                           R.rw.p, R.kappa.p,
                                                                           rl_[size_t(l + 1)].kappa.p);
        kr_weights<<<rgrid(L.n), kRThreads, 0, s>>>(L.n, L.rowptr.p, L.col.p, L.d.val.p, L.ncomp > 0 ? 1 : 0,
                                                   L.d.dinv.p, L.f.dinv.p, l + 1 < nl ? L.d.tinv.p : nullptr,
                                                   l + 1 < nl ? L.f.tinv.p : nullptr, rpart_.p, rcnt_.p,
                                                   rwtw_.p + 2 * l, rerr_.p);
    }
    const DevLevel& C = levels_.back();
    TPA_CUDA(cudaMemsetAsync(coarse_M_.p, 0, sizeof(double) * coarse_M_.n, s));
    kr_coarse_fill<<<rgrid(C.n), kRThreads, 0, s>>>(C.n, coarse_N_, C.rowptr.p, C.col.p, C.d.val.p,
                                                   coarse_ncomp_ > 0 ? C.slot.p : nullptr, C.d.vol.p, coarse_ncomp_,
                                                   coarse_M_.p);
    const int N = coarse_N_;
    const size_t cl_bytes = (size_t((N + kLuCluster - 1) / kLuCluster) * N + 2 * size_t(N)) * sizeof(double);
    if (lu_cluster_) {
        cudaLaunchConfig_t cfg;
        std::memset(&cfg, 0, sizeof(cfg));
        cfg.gridDim = dim3(kLuCluster);
        cfg.blockDim = dim3(kLuClusterThreads);
        cfg.dynamicSmemBytes = cl_bytes;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = kLuCluster;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        TPA_CUDA(cudaLaunchKernelEx(&cfg, kr_lu<true>, N, coarse_M_.p, coarse_piv_.p, rerr_.p));
    } else {
        kr_lu<false><<<1, 1024, 2 * size_t(N) * sizeof(double), s>>>(N, coarse_M_.p, coarse_piv_.p, rerr_.p);
    }
    const size_t inv_bytes = size_t(kInvWarps) * size_t(N) * sizeof(double);
    kr_coarse_inv<<<(C.n + kInvWarps - 1) / kInvWarps, 32 * kInvWarps, inv_bytes, s>>>(N, C.n, coarse_M_.p,
                                                                                     coarse_piv_.p, coarse_inv_.p, rerr_.p);
    TPA_CUDA(cudaGetLastError());
    std::vector<double> wtw(size_t(2 * nl));
    int err = 0;
    TPA_CUDA(cudaMemcpyAsync(wtw.data(), rwtw_.p, sizeof(double) * wtw.size(), cudaMemcpyDeviceToHost, s));
    TPA_CUDA(cudaMemcpyAsync(&err, rerr_.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    TPA_CUDA(cudaStreamSynchronize(s));
    if (err == 1) throw Error(1, "elliptic matrix has a non-positive diagonal");
    if (err == 2) throw Error(1, "coarsest multigrid matrix is singular");
    for (int l = 0; l < nl; ++l) {
        DevLevel& L = levels_[size_t(l)];
        L.d.w = wtw[size_t(2 * l)];
        L.f.w = float(L.d.w);
        if (l + 1 < nl) {
            L.d.tw = wtw[size_t(2 * l + 1)];
            L.f.tw = float(L.d.tw);
        }
        vd_[size_t(l)].w = L.d.w;
        vf_[size_t(l)].w = L.f.w;
        vd_[size_t(l)].tw = L.d.tw;
        vf_[size_t(l)].tw = L.f.tw;
    }
    // the level views (and the captured graphs, which hold them by value) change
    vd_dev_.upload(vd_.data(), vd_.size(), s);
    vf_dev_.upload(vf_.data(), vf_.size(), s);
    TPA_CUDA(cudaStreamSynchronize(s));
    destroy_graphs();
    invalidate_faces();
}

std::vector<double> DeviceSolver::level_weights() {
    std::vector<double> out;
    for (const DevLevel& L : levels_) {
        out.push_back(L.d.w);
        out.push_back(L.d.tw);
    }
    return out;
}

}  // namespace tpa
