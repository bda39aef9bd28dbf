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
#include "structure.hpp"

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

// new coefficients against the current ones: flags |= 1 for a value that is
// not finite or negative, |= 2 where the set of zero coefficients differs
__global__ void kr_check(int n, const double* __restrict__ k_new, const double* __restrict__ k_old, int* flags) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = k_new[i];
        if (!(isfinite(v) && v >= 0.0)) atomicOr(flags, 1);
        else if ((v == 0.0) != (k_old[i] == 0.0)) atomicOr(flags, 2);
    }
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

// D^-1 and Dt^-1 per row and the Jacobi bounds max_i sum_j |a_ij| / a_ii;
// the last block writes w = min(1, 4/(3 bound)) (1 without a bound), the
// unclamped transfer weight 4/(3 bound) (0 without a bound) and, with a
// red-black colouring, the half-sweep weight from the rows restricted to their
// own colour into wtw[0..2].
__global__ void kr_weights(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ val, int singular, const unsigned char* __restrict__ colour,
                           double* __restrict__ dinv_d, float* __restrict__ dinv_f, double* __restrict__ tinv_d,
                           float* __restrict__ tinv_f, double* partial, unsigned* counter, double* wtw, int* err) {
    double bs = 0.0, bt = 0.0, br = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double d = 0.0, rs = 0.0, rc = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            rs += fabs(val[k]);
            if (ci[k] == i) d = val[k];
            if (colour && colour[ci[k]] == colour[i]) rc += fabs(val[k]);
        }
        if (d > 0) br = fmax(br, rc / d);
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
    __shared__ double sh[3][32];
    __shared__ bool last;
    for (int o = 16; o; o >>= 1) {
        bs = fmax(bs, __shfl_down_sync(0xffffffffu, bs, o));
        bt = fmax(bt, __shfl_down_sync(0xffffffffu, bt, o));
        br = fmax(br, __shfl_down_sync(0xffffffffu, br, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (!lane) {
        sh[0][wid] = bs;
        sh[1][wid] = bt;
        sh[2][wid] = br;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ms = 0.0, mt = 0.0, mr = 0.0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) {
            ms = fmax(ms, sh[0][w]);
            mt = fmax(mt, sh[1][w]);
            mr = fmax(mr, sh[2][w]);
        }
        partial[blockIdx.x] = ms;
        partial[gridDim.x + blockIdx.x] = mt;
        partial[2 * gridDim.x + blockIdx.x] = mr;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double ms = 0.0, mt = 0.0, mr = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) {
            ms = fmax(ms, ((volatile double*)partial)[b]);
            mt = fmax(mt, ((volatile double*)partial)[gridDim.x + b]);
            mr = fmax(mr, ((volatile double*)partial)[2 * gridDim.x + b]);
        }
        wtw[0] = ms == 0.0 ? 1.0 : fmin(1.0, 4.0 / (3.0 * ms));
        wtw[1] = mt == 0.0 ? 0.0 : 4.0 / (3.0 * mt);
        wtw[2] = mr == 0.0 ? 1.0 : fmin(1.0, 4.0 / (3.0 * mr));
        *counter = 0;
    }
}

// stencil copies of a block-structured level: east / north couplings -a_ij
// gathered from the refreshed operator (0 where the entry is absent)
__global__ void kr_gather_stencil(int n, const int* __restrict__ px, const int* __restrict__ py,
                                  const double* __restrict__ val, double* __restrict__ cx_d, float* __restrict__ cx_f,
                                  double* __restrict__ cy_d, float* __restrict__ cy_f) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double cx = px[i] >= 0 ? -val[px[i]] : 0.0, cy = py[i] >= 0 ? -val[py[i]] : 0.0;
        cx_d[i] = cx;
        cx_f[i] = float(cx);
        cy_d[i] = cy;
        cy_f[i] = float(cy);
    }
}

// the exception rows' values (their CSR entries in row order)
__global__ void kr_gather(int m, const int* __restrict__ pos, const double* __restrict__ val,
                          double* __restrict__ out_d, float* __restrict__ out_f) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const double v = val[pos[k]];
        out_d[k] = v;
        out_f[k] = float(v);
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

constexpr int kLuMaxCluster = 8;

// LU with partial pivoting of the augmented coarsest matrix M (N x N,
// row-major, overwritten by the factors; piv[k] = row exchanged with row k).
// Cl: the rows are spread cyclically over the C CTAs of a thread-block cluster
// (row r on CTA r % C at local row r / C) and held in shared memory; otherwise
// one CTA works on M in global memory (C = 1).  Each step follows the host
// factorisation operation for operation: the pivot is the first row of largest
// |M[r][k]| (r >= k), rows k and p are exchanged whole, l = M[r][k] *
// (1 / M[k][k]) overwrites M[r][k] and M[r][c] -= l M[k][c] (c > k, l != 0).
//
// One cluster barrier per step: after its update every CTA pushes its best
// candidate for the next pivot -- value, row and the whole row -- into the
// shared memory of every CTA, and the owner of row k + 1 pushes that row too,
// so the next step picks the pivot and exchanges rows from local copies.  The
// push buffers alternate between two sets (a step reads one while the pushes
// for the next fill the other).  err = 2 on a zero pivot.
template <bool Cl>
__global__ void __launch_bounds__(1024) kr_lu(int N, double* __restrict__ M, int* __restrict__ piv, int* err) {
    namespace cg = cooperative_groups;
    extern __shared__ double lu_sm[];
    __shared__ double wv[32];
    __shared__ int wi[32];
    __shared__ double cval[2][kLuMaxCluster];
    __shared__ int cidx[2][kLuMaxCluster];
    int C = 1, rank = 0;
    if constexpr (Cl) {
        C = int(cg::this_cluster().num_blocks());
        rank = int(cg::this_cluster().block_rank());
    }
    const int R = (N + C - 1) / C;
    double* rows = Cl ? lu_sm : M;
    double* cbuf = Cl ? lu_sm + size_t(R) * N : lu_sm;  // [2][C][N] candidate rows by source
    double* kbuf = cbuf + size_t(2) * C * N;             // [2][N] row k before the exchange
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = int(blockDim.x >> 5);
    // the same shared-memory word in CTA q of the cluster (this CTA's own for C = 1)
    auto peer = [&](auto* ptr, int q) {
        if constexpr (Cl) return cg::this_cluster().map_shared_rank(ptr, q);
        else return ptr;
    };
    const size_t cb_off = size_t(cbuf - lu_sm), kb_off = size_t(kbuf - lu_sm);
    auto first_local = [&](int j) {  // smallest local row whose global row is >= j
        const int t = j - rank;
        return t <= 0 ? 0 : (t + C - 1) / C;
    };
    // CTA-wide best (value, row); every thread returns the same pair
    auto reduce = [&](double bv, int bi, double& v, int& i) {
        for (int o = 16; o; o >>= 1) better(bv, bi, __shfl_down_sync(0xffffffffu, bv, o),
                                            __shfl_down_sync(0xffffffffu, bi, o));
        if (!lane) {
            wv[wid] = bv;
            wi[wid] = bi;
        }
        __syncthreads();
        v = lane < nw ? wv[lane] : -1.0;
        i = lane < nw ? wi[lane] : N;
        for (int o = 16; o; o >>= 1) better(v, i, __shfl_xor_sync(0xffffffffu, v, o), __shfl_xor_sync(0xffffffffu, i, o));
    };
    // the candidate (v, i) and row i, and row j if this CTA owns it, into set b everywhere
    auto push = [&](int b, double v, int i, int j) {
        if (threadIdx.x < C) {
            *peer(&cval[b][rank], int(threadIdx.x)) = v;
            *peer(&cidx[b][rank], int(threadIdx.x)) = i;
        }
        if (i < N) {
            const double* src = rows + size_t(i / C) * N;
            const size_t off = cb_off + (size_t(b) * C + rank) * N;
            for (int c = threadIdx.x; c < N; c += blockDim.x) {
                const double x = src[c];
                for (int q = 0; q < C; ++q) *peer(lu_sm + off + c, q) = x;
            }
        }
        if (j < N && j % C == rank) {
            const double* src = rows + size_t(j / C) * N;
            const size_t off = kb_off + size_t(b) * N;
            for (int c = threadIdx.x; c < N; c += blockDim.x) {
                const double x = src[c];
                for (int q = 0; q < C; ++q) *peer(lu_sm + off + c, q) = x;
            }
        }
    };
    if constexpr (Cl) {
        for (int lr = 0; lr < R && lr * C + rank < N; ++lr)
            for (int c = threadIdx.x; c < N; c += blockDim.x)
                rows[size_t(lr) * N + c] = M[size_t(lr * C + rank) * N + c];
        __syncthreads();
    }
    {
        double bv = -1.0, v;
        int bi = N, i;
        for (int lr = first_local(0) + int(threadIdx.x); lr < R && lr * C + rank < N; lr += blockDim.x)
            better(bv, bi, fabs(rows[size_t(lr) * N]), lr * C + rank);
        reduce(bv, bi, v, i);
        push(0, v, i, 0);
    }
    lu_sync<Cl>();
    for (int k = 0; k < N; ++k) {
        const int b = k & 1;
        // lane q of every group of eight holds the candidate pushed by CTA q
        const int q8 = lane & (kLuMaxCluster - 1);
        double v = q8 < C ? cval[b][q8] : -1.0;
        int p = q8 < C ? cidx[b][q8] : N;
        for (int o = 4; o; o >>= 1) better(v, p, __shfl_xor_sync(0xffffffffu, v, o), __shfl_xor_sync(0xffffffffu, p, o));
        const int src = p % C;  // the owner of row p pushed it
        if (!(v > 0.0) || p >= N) {  // every CTA takes the same decision
            if (rank == 0 && threadIdx.x == 0) atomicExch(err, 2);
            break;
        }
        if (rank == 0 && threadIdx.x == 0) piv[k] = p;
        const double* prow = cbuf + (size_t(b) * C + src) * N;
        const double* krow = kbuf + size_t(b) * N;
        if (p != k) {
            if (rank == k % C)
                for (int c = threadIdx.x; c < N; c += blockDim.x) rows[size_t(k / C) * N + c] = prow[c];
            if (rank == p % C)
                for (int c = threadIdx.x; c < N; c += blockDim.x) rows[size_t(p / C) * N + c] = krow[c];
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
        double nv;
        int ni;
        reduce(bv, bi, nv, ni);  // its barrier also orders the updates before the pushes
        if (k + 1 < N) push(b ^ 1, nv, ni, k + 1);
        lu_sync<Cl>();
    }
    lu_sync<Cl>();  // no CTA leaves while another may still write into its buffers
    if constexpr (Cl) {
        for (int lr = 0; lr < R && lr * C + rank < N; ++lr)
            for (int c = threadIdx.x; c < N; c += blockDim.x)
                M[size_t(lr * C + rank) * N + c] = rows[size_t(lr) * N + c];
    }
}

// Shared memory (bytes) of kr_lu: rows (cluster form only), two sets of C
// candidate rows and two copies of row k.
size_t lu_smem(int N, int C, bool cluster) {
    const size_t R = size_t((N + C - 1) / C);
    return ((cluster ? R * size_t(N) : 0) + 2 * size_t(C) * N + 2 * size_t(N)) * sizeof(double);
}

constexpr int kInvWarps = 4;  // columns of the inverse per CTA

// MT = M' (the factors by columns), 32 x 32 tiles through shared memory
__global__ void kr_transpose(int N, const double* __restrict__ M, double* __restrict__ MT, const int* err) {
    __shared__ double tile[32][33];
    if (*err) return;
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = by + j, c = bx + int(threadIdx.x);
        if (r < N && c < N) tile[j][threadIdx.x] = M[size_t(r) * N + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = bx + j, c = by + int(threadIdx.x);
        if (r < N && c < N) MT[size_t(r) * N + c] = tile[threadIdx.x][j];
    }
}

// The first n columns of M^-1 from the factors, one warp per column, in
// blocks of 32 rows: lane t owns row 32 B + t.  A block first subtracts the
// solved blocks' contribution (lane t reads MT[k][32 B + t]: consecutive
// addresses across the warp), then resolves its own 32 rows in order with the
// solved value broadcast by a shuffle.  Forward with the unit lower factor
// from the permuted unit vector (blocks above its 1 stay zero), back with the
// upper factor; G[r][col] = e[r] for r < n.  The order of each row's sum is
// fixed (deterministic).
__global__ void __launch_bounds__(32 * kInvWarps) kr_coarse_inv(int N, int n, const double* __restrict__ MT,
                                                               const int* __restrict__ piv,
                                                               double* __restrict__ G,
                                                               const int* __restrict__ err) {
    extern __shared__ double inv_sm[];
    if (*err) return;  // uniform over the grid
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int col = int(blockIdx.x) * kInvWarps + wid;
    if (col >= n) return;  // whole warps; no block-wide barrier follows
    double* e = inv_sm + size_t(wid) * N;
    int pos = col;
    for (int k = 0; k < N; ++k) {
        const int p = piv[k];
        if (pos == k) pos = p;
        else if (pos == p) pos = k;
    }
    const int nb = (N + 31) / 32;
    // sum over k in [k0, k1) of MT[k][r] e[k]: four interleaved partial sums,
    // combined in a fixed order (the loads of a row run ahead of its FMAs)
    auto dot = [&](int r, int k0, int k1) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int k = k0;
        for (; k + 4 <= k1; k += 4) {
            s0 += MT[size_t(k) * N + r] * e[k];
            s1 += MT[size_t(k + 1) * N + r] * e[k + 1];
            s2 += MT[size_t(k + 2) * N + r] * e[k + 2];
            s3 += MT[size_t(k + 3) * N + r] * e[k + 3];
        }
        for (; k < k1; ++k) s0 += MT[size_t(k) * N + r] * e[k];
        return (s0 + s1) + (s2 + s3);
    };
    // the block's 32 x 32 tile of the factor in registers: lane t holds
    // M[32 B + t][32 B + kk] in t[kk] (0 beyond N)
    double tile[32];
    auto load_tile = [&](int B, int r, bool ok) {
#pragma unroll
        for (int kk = 0; kk < 32; ++kk) {
            const int k = 32 * B + kk;
            tile[kk] = (ok && k < N) ? MT[size_t(k) * N + r] : 0.0;
        }
    };
    // forward: L y = P e_col
    for (int k = lane; k < N; k += 32) e[k] = 0.0;
    __syncwarp();
    for (int B = pos / 32; B < nb; ++B) {
        const int r = 32 * B + lane;
        const bool ok = r < N;
        load_tile(B, r, ok);
        double v = (r == pos) ? 1.0 : 0.0;
        if (ok) v -= dot(r, (pos / 32) * 32, 32 * B);
#pragma unroll
        for (int kk = 0; kk < 32; ++kk) {
            const double ek = __shfl_sync(0xffffffffu, v, kk);
            if (lane > kk) v -= tile[kk] * ek;
        }
        if (ok) e[r] = v;
        __syncwarp();
    }
    // backward: U x = y (lane kk's tile[kk] is the diagonal U[k][k])
    for (int B = nb - 1; B >= 0; --B) {
        const int r = 32 * B + lane;
        const bool ok = r < N;
        load_tile(B, r, ok);
        double v = ok ? e[r] : 0.0;
        if (ok) v -= dot(r, 32 * (B + 1), N);
#pragma unroll
        for (int kk = 31; kk >= 0; --kk) {
            if (32 * B + kk < N) {  // uniform over the warp
                if (lane == kk) v = v / tile[kk];
                const double ek = __shfl_sync(0xffffffffu, v, kk);
                if (lane < kk) v -= tile[kk] * ek;
            }
        }
        if (ok) e[r] = v;
        __syncwarp();
    }
    for (int r = lane; r < n; r += 32) G[size_t(r) * n + col] = e[r];
}

size_t inv_smem(int N) { return size_t(kInvWarps) * size_t(N) * sizeof(double); }

constexpr int kLuCluster = 8;  // CTAs sharing the rows of the coarsest matrix
constexpr int kLuClusterThreads = 512;

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
        if (l == 0 && nf > 0)  // the current coefficients: the zero-set check of a device refresh
            R.kappa.upload(op.kappa.data(), op.kappa.size(), stream_);
        R.sk.alloc(size_t(std::max<int64_t>(nf, 1)));
        const HostLevel& hl = h.levels[size_t(l)];
        if (size_t(l) < sdev_.size() && sdev_[size_t(l)].on) {
            // the same block structure as the stencil copies (upload_structured)
            const StructLevel st = build_struct(hl, &h.levels[size_t(l + 1)].op.mesh);
            const int nx = st.nx, ny = st.ny, cpb = nx * ny;
            auto neighbour = [&](int64_t c, int d) -> int64_t {  // 0 W, 1 E, 2 S, 3 N
                const int64_t b = c / cpb, r = c % cpb;
                int i = int(r % nx) + (d == 0 ? -1 : d == 1 ? 1 : 0), j = int(r / nx) + (d == 2 ? -1 : d == 3 ? 1 : 0);
                if (i >= 0 && i < nx && j >= 0 && j < ny) return b * cpb + j * nx + i;
                const int32_t q = st.nbr[size_t(4 * b + d)];
                if (q < 0) return -1;
                return int64_t(q) * cpb + ((j + ny) % ny) * nx + (i + nx) % nx;
            };
            auto at = [&](int64_t r, int64_t c) -> int {
                if (c < 0) return -1;
                auto b = A.col.begin() + A.ptr[size_t(r)], e = A.col.begin() + A.ptr[size_t(r + 1)];
                auto it = std::lower_bound(b, e, int32_t(c));
                return (it == e || *it != c) ? -1 : int(it - A.col.begin());
            };
            std::vector<int> px(size_t(A.n)), py(size_t(A.n)), sex;
            for (int64_t c = 0; c < A.n; ++c) {
                px[size_t(c)] = at(c, neighbour(c, 1));
                py[size_t(c)] = at(c, neighbour(c, 3));
                if (st.ex[size_t(c)] >= 0)
                    for (int64_t k = A.ptr[size_t(c)]; k < A.ptr[size_t(c + 1)]; ++k) sex.push_back(int(k));
            }
            if (int64_t(sex.size()) != int64_t(st.ex_val.size()))
                throw Error(7, "exception rows of the device refresh disagree with the stencil copies");
            R.structured = true;
            R.nex_entries = int(sex.size());
            R.sx.upload(px.data(), px.size(), stream_);
            R.sy.upload(py.data(), py.size(), stream_);
            R.sex.upload(sex.data(), sex.size(), stream_);
            TPA_CUDA(cudaStreamSynchronize(stream_));
        }
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
    coarse_MT_.alloc(size_t(coarse_N_) * size_t(coarse_N_));
    {
        // the cluster LU when a cluster's shared memory holds the matrix
        const int N = coarse_N_;
        int optin = 0;
        TPA_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device_));
        const size_t room = size_t(optin) - 1024;  // static shared memory of the kernels
        const size_t cl_bytes = lu_smem(N, kLuCluster, true);
        lu_cluster_ = cl_bytes <= room && !std::getenv("TPAGMG_LU_ONE_CTA");
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
        const size_t one_bytes = lu_smem(N, 1, false), inv_bytes = inv_smem(N);
        if (one_bytes > room || inv_bytes > room) throw Error(5, "coarsest matrix too large for the device refresh");
        TPA_CUDA(cudaFuncSetAttribute(kr_lu<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(one_bytes)));
        TPA_CUDA(cudaFuncSetAttribute(kr_coarse_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, int(inv_bytes)));
    }
    coarse_piv_.alloc(size_t(coarse_N_));
    if (rstage_) cudaFreeHost(rstage_);
    rstage_ = nullptr;
    TPA_CUDA(cudaMallocHost(&rstage_, sizeof(double) * std::max<size_t>(1, size_t(rl_[0].nf))));
    rwtw_.alloc(size_t(3 * nl));
    rpart_.alloc(size_t(3 * 1184));
    rcnt_.alloc(1);
    rerr_.alloc(1);
    TPA_CUDA(cudaMemsetAsync(rcnt_.p, 0, sizeof(unsigned), stream_));
    TPA_CUDA(cudaMemsetAsync(coarse_piv_.p, 0, sizeof(int) * coarse_piv_.n, stream_));
    TPA_CUDA(cudaStreamSynchronize(stream_));
    rl_ready_ = true;
}

bool DeviceSolver::refresh_applicable(const Hierarchy& h) const {
    // the entry term lists hold the face couplings only; levels with open-face
    // conductances on their diagonal are refreshed on the host
    for (const HostLevel& l : h.levels)
        if (l.op.any_open()) return false;
    // stencil copies are gathered from the refreshed operator; a level kept as
    // one constant coupling or diagonal would change layout, so it needs the host
    for (const StructDev& D : sdev_)
        if (D.on && (D.const_coef || D.const_diag)) return false;
    const HostLevel& c = h.levels.back();
    const int64_t N = c.op.A.n + (c.op.singular ? int64_t(c.op.comp.volume.size()) : 0);
    return N <= kRefreshMaxCoarse;
}

void DeviceSolver::refresh_on_device(const Hierarchy& h, const double* kappa_host) {
    TPA_CUDA(cudaSetDevice(device_));
    if (!rl_ready_) prepare_refresh(h);
    std::memcpy(rstage_, kappa_host, sizeof(double) * size_t(rl_[0].nf));  // no copy is in flight here
    TPA_CUDA(cudaMemcpyAsync(rl_[0].kappa.p, rstage_, sizeof(double) * size_t(rl_[0].nf), cudaMemcpyHostToDevice,
                             stream_));
    refresh_levels();
}

int DeviceSolver::refresh_from_device(const Hierarchy& h, const double* kappa_dev) {
    TPA_CUDA(cudaSetDevice(device_));
    if (!rl_ready_) prepare_refresh(h);
    const int nf = rl_[0].nf;
    int flags = 0;
    TPA_CUDA(cudaMemsetAsync(rerr_.p, 0, sizeof(int), stream_));
    if (nf > 0) kr_check<<<rgrid(nf), kRThreads, 0, stream_>>>(nf, kappa_dev, rl_[0].kappa.p, rerr_.p);
    TPA_CUDA(cudaMemcpyAsync(&flags, rerr_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    TPA_CUDA(cudaStreamSynchronize(stream_));
    if (flags & 1) throw Error(1, "face coefficients must be finite and nonnegative");
    if (flags & 2) return 1;
    TPA_CUDA(cudaMemcpyAsync(rl_[0].kappa.p, kappa_dev, sizeof(double) * size_t(nf), cudaMemcpyDeviceToDevice,
                             stream_));
    refresh_levels();
    return 0;
}

void DeviceSolver::refresh_levels() {
    const int nl = int(levels_.size());
    cudaStream_t s = stream_;
    TPA_CUDA(cudaMemsetAsync(rerr_.p, 0, sizeof(int), s));
    for (int l = 0; l < nl; ++l) {
        RefreshLevel& R = rl_[size_t(l)];
        DevLevel& L = levels_[size_t(l)];
        if (R.nf > 0) kr_sqrt<<<rgrid(R.nf), kRThreads, 0, s>>>(R.nf, R.kappa.p, R.sk.p);
        kr_assemble<<<rgrid(R.nnz), kRThreads, 0, s>>>(R.nnz, R.tptr.p, R.tf.p, R.tg.p, R.tc.p, R.kappa.p, R.sk.p,
                                                      L.d.val.p, L.f.val.p);
        if (R.structured) {
            StructDev& D = sdev_[size_t(l)];
            kr_gather_stencil<<<rgrid(L.n), kRThreads, 0, s>>>(L.n, R.sx.p, R.sy.p, L.d.val.p, D.cx_d.p, D.cx_f.p,
                                                               D.cy_d.p, D.cy_f.p);
            if (R.nex_entries)
                kr_gather<<<rgrid(R.nex_entries), kRThreads, 0, s>>>(R.nex_entries, R.sex.p, L.d.val.p, D.exv_d.p,
                                                                     D.exv_f.p);
        }
        if (l + 1 < nl && rl_[size_t(l + 1)].nf > 0)
            kr_restrict<<<rgrid(rl_[size_t(l + 1)].nf), kRThreads, 0, s>>>(rl_[size_t(l + 1)].nf, R.rptr.p, R.ridx.p,
                                                                           R.rw.p, R.kappa.p,
                                                                           rl_[size_t(l + 1)].kappa.p);
        kr_weights<<<rgrid(L.n), kRThreads, 0, s>>>(L.n, L.rowptr.p, L.col.p, L.d.val.p, L.ncomp > 0 ? 1 : 0,
                                                   rb_ ? L.colour.p : nullptr,
                                                   L.d.dinv.p, L.f.dinv.p, l + 1 < nl ? L.d.tinv.p : nullptr,
                                                   l + 1 < nl ? L.f.tinv.p : nullptr, rpart_.p, rcnt_.p,
                                                   rwtw_.p + 3 * l, rerr_.p);
    }
    const DevLevel& C = levels_.back();
    TPA_CUDA(cudaMemsetAsync(coarse_M_.p, 0, sizeof(double) * coarse_M_.n, s));
    kr_coarse_fill<<<rgrid(C.n), kRThreads, 0, s>>>(C.n, coarse_N_, C.rowptr.p, C.col.p, C.d.val.p,
                                                   coarse_ncomp_ > 0 ? C.slot.p : nullptr, C.d.vol.p, coarse_ncomp_,
                                                   coarse_M_.p);
    const int N = coarse_N_;
    if (lu_cluster_) {
        cudaLaunchConfig_t cfg;
        std::memset(&cfg, 0, sizeof(cfg));
        cfg.gridDim = dim3(kLuCluster);
        cfg.blockDim = dim3(kLuClusterThreads);
        cfg.dynamicSmemBytes = lu_smem(N, kLuCluster, true);
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
        kr_lu<false><<<1, 1024, lu_smem(N, 1, false), s>>>(N, coarse_M_.p, coarse_piv_.p, rerr_.p);
    }
    {
        const dim3 tg((N + 31) / 32, (N + 31) / 32), tb(32, 8);
        kr_transpose<<<tg, tb, 0, s>>>(N, coarse_M_.p, coarse_MT_.p, rerr_.p);
    }
    kr_coarse_inv<<<(C.n + kInvWarps - 1) / kInvWarps, 32 * kInvWarps, inv_smem(N), s>>>(
        N, C.n, coarse_MT_.p, coarse_piv_.p, coarse_inv_.p, rerr_.p);
    TPA_CUDA(cudaGetLastError());
    std::vector<double> wtw(size_t(3 * nl));
    int err = 0;
    TPA_CUDA(cudaMemcpyAsync(wtw.data(), rwtw_.p, sizeof(double) * wtw.size(), cudaMemcpyDeviceToHost, s));
    TPA_CUDA(cudaMemcpyAsync(&err, rerr_.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    TPA_CUDA(cudaStreamSynchronize(s));
    if (err == 1) throw Error(1, "elliptic matrix has a non-positive diagonal");
    if (err == 2) throw Error(1, "coarsest multigrid matrix is singular");
    for (int l = 0; l < nl; ++l) {
        DevLevel& L = levels_[size_t(l)];
        L.d.w = wtw[size_t(3 * l)];
        L.f.w = float(L.d.w);
        if (l + 1 < nl) {
            L.d.tw = wtw[size_t(3 * l + 1)];
            L.f.tw = float(L.d.tw);
        }
        if (rb_) {
            L.rbw = wtw[size_t(3 * l + 2)];
            vd_[size_t(l)].rbw = L.rbw;
            vf_[size_t(l)].rbw = float(L.rbw);
        }
        vd_[size_t(l)].w = L.d.w;
        vf_[size_t(l)].w = L.f.w;
        vd_[size_t(l)].tw = L.d.tw;
        vf_[size_t(l)].tw = L.f.tw;
        if (size_t(l) < sd_.size()) {
            sd_[size_t(l)].w = L.d.w;
            sf_[size_t(l)].w = L.f.w;
            sd_[size_t(l)].tw = L.d.tw;
            sf_[size_t(l)].tw = L.f.tw;
        }
    }
    // the level views (and the captured graphs, which hold them by value) change
    vd_dev_.upload(vd_.data(), vd_.size(), s);
    vf_dev_.upload(vf_.data(), vf_.size(), s);
    // the face kernels' sqrt(kappa) (same faces, same zero set)
    if (nfaces_ >= 0 && rl_[0].nf > 0)
        TPA_CUDA(cudaMemcpyAsync(f_sqrtk_.p, rl_[0].sk.p, sizeof(double) * size_t(rl_[0].nf), cudaMemcpyDeviceToDevice,
                                 s));
    TPA_CUDA(cudaStreamSynchronize(s));
    gather_tile_values();  // the tile copies of the refreshed level values
    destroy_graphs();
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
