// Fused per-level V-cycle kernels on haloed block tiles (tiles.hpp).
//
// A level of the default cycle (damped Jacobi, two pre- and two post-sweeps,
// src/solvers/multigrid/cycles.jl:8-77 of ronaldremmerswaal/TwoPhaseAMR.jl)
// costs six dependent launches on the unfused path (k_pre2, k_residual,
// k_restrict, k_prolong, k_post1, k_post2).  Here one CTA owns one block and
// recomputes the values its block needs from a halo of three rings, so a
// level costs two launches:
//   k_tile_down  rings <= 3: x1 = w D^-1 bp (the first sweep from zero);
//                rings <= 2: x2 = x1 + w D^-1 (bp - A x1);
//                rings <= 1: r = bp - A x2, s = Dt^-1 r;
//                the block:  b_c = P_tent'(r - wt A s) for its coarse cells,
//                            x2 and bp stored (x2 into L.y), the coarse RHS sum
//   k_tile_up    rings <= 3: e = x_c(owner);
//                rings <= 2: x = x2 + e - wt Dt^-1 A e;
//                rings <= 1: x' = x + w D^-1 (bp - A x);
//                the block:  x'' = x' + w D^-1 (bp - A x') into L.x, the
//                            finest level's mean (and epilogue)
// Every row is summed in CSR order with the arithmetic of the unfused kernels
// (pre2_cell, residual_cell, restrict_quad, prolong_cell, sweep_cell), so the
// two paths give the same V-cycle up to the order of the coarse RHS sum.
#pragma once

#include <cuda_runtime.h>

#include "fused.cuh"
#include "stencil.cuh"

namespace tpa {

constexpr int kTileThreads = 256;  // stencil tiles; CSR tiles take NT = 256, 512 or 1024
constexpr int kTileMaxCells = 1536;  // cells of a CSR tile (rings <= 3) at most

// One level's tiles in precision T (device pointers).
template <typename T>
struct TileView {
    int ntiles;
    int n3max, n2max, n1max, emax;
    const int* cell;
    const int* own;    // parallel to cell: tentative owner on the coarse level
    const int* cell_off;
    const int4* ring;  // per tile: cells of rings <= 0, 1, 2, 3
    const int* lrp;
    const int* lrp_off;
    const int* ent_off;
    const T* val;      // the level's CSR values in tile entry order
    const short* lcol;
    const int* co;
    const int* co_off;
    const short4* ch;  // per coarse cell: local indices of its children (-1: none)
};

// Shared memory of a tile: the cell arrays in precision T, the tile's CSR
// values (T), its local row pointers (int) and local columns (short), so that
// every phase after the prologue reads shared memory only.
template <typename T>
__host__ __device__ inline size_t tile_down_smem(int n3, int n2, int n1, int e) {
    return sizeof(T) * (3 * size_t(n3) + size_t(n2) + 3 * size_t(n1) + size_t(e)) + sizeof(int) * (size_t(n2) + 1) +
           sizeof(short) * size_t(e);
}

template <typename T>
__host__ __device__ inline size_t tile_up_smem(int n3, int n2, int n1, int e) {
    return sizeof(T) * (size_t(n3) + 3 * size_t(n2) + 2 * size_t(n1) + size_t(e)) + sizeof(int) * (size_t(n2) + 1) +
           sizeof(short) * size_t(e);
}

// Loads in flight per thread in the prologues: a CTA's latency is that of its
// dependent load chains, so every batch of independent loads is issued before
// any of them is used.
constexpr int kTileEntriesPerThread = 8;

// the tile's local CSR into shared memory (coalesced copies, 8 entries in flight)
template <typename T, int NT>
__device__ __forceinline__ void tile_stage_csr(const TileView<T>& V, int t, int n2, T* sval, int* slrp, short* slc) {
    const int* rowp = V.lrp + V.lrp_off[t];
    const int e0 = V.ent_off[t], ne = V.ent_off[t + 1] - e0;
    const T* val = V.val + e0;
    const short* lc = V.lcol + e0;
    constexpr int U = kTileEntriesPerThread;
    for (int base = threadIdx.x; base < ne; base += U * NT) {
        T v[U];
        short c[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = base + u * NT;
            if (e < ne) {
                v[u] = val[e];
                c[u] = lc[e];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = base + u * NT;
            if (e < ne) {
                sval[e] = v[u];
                slc[e] = c[u];
            }
        }
    }
    for (int k = threadIdx.x; k <= n2; k += blockDim.x) slrp[k] = rowp[k];
}

template <typename T>
__device__ __forceinline__ T tile_rowdot(const T* val, const short* lc, const int* lrp, const T* v, int k) {
    T acc = T(0);
    for (int e = lrp[k]; e < lrp[k + 1]; ++e) acc += val[e] * v[lc[e]];
    return acc;
}

__device__ __forceinline__ int short4_at(short4 v, int q) {
    return q == 0 ? v.x : q == 1 ? v.y : q == 2 ? v.z : v.w;
}

// b: this level's raw right-hand side (the FP64 residual on the finest level);
// level_sum: its sum (projection, may be null); bc: the coarse right-hand side;
// coarse_sum (may be null): receives the sum of bc, folded by the last CTA.
template <typename T, typename TB, int NT>
__global__ void __launch_bounds__(NT)
    k_tile_down(LevelView<T> L, TileView<T> V, const TB* __restrict__ b, const double* level_sum,
                T* __restrict__ bc, double* partial, unsigned* counter, double* coarse_sum) {
    pdl_entry();
    extern __shared__ __align__(16) unsigned char tile_smem[];
    T* bp = reinterpret_cast<T*>(tile_smem);
    T* dv = bp + V.n3max;
    T* xa = dv + V.n3max;
    T* xb = xa + V.n3max;
    T* ti = xb + V.n2max;
    T* rr = ti + V.n1max;
    T* ss = rr + V.n1max;
    T* val = ss + V.n1max;
    int* lrp = reinterpret_cast<int*>(val + V.emax);
    short* lc = reinterpret_cast<short*>(lrp + V.n2max + 1);
    const int t = blockIdx.x;
    const int4 R = V.ring[t];
    const int* cell = V.cell + V.cell_off[t];
    constexpr int CU = (kTileMaxCells + NT - 1) / NT;
    int g[CU];
#pragma unroll
    for (int u = 0; u < CU; ++u) {
        const int k = threadIdx.x + u * NT;
        g[u] = k < R.w ? cell[k] : -1;
    }
    tile_stage_csr<T, NT>(V, t, R.z, val, lrp, lc);
    const double mean = (L.singular && level_sum) ? *level_sum * L.cvol_inv : 0.0;
    TB bb[CU];
    T vv[CU], dd[CU], tt[CU];
#pragma unroll
    for (int u = 0; u < CU; ++u) {
        if (g[u] >= 0) {
            bb[u] = b[g[u]];
            vv[u] = L.singular ? L.vol[g[u]] : T(0);
            dd[u] = L.dinv[g[u]];
            tt[u] = L.tinv[g[u]];
        }
    }
#pragma unroll
    for (int u = 0; u < CU; ++u) {
        const int k = threadIdx.x + u * NT;
        if (g[u] >= 0) {
            // the projected RHS as proj_b forms it
            double v = double(bb[u]);
            if (L.singular) v -= double(vv[u]) * mean;
            const T bk = T(v);
            bp[k] = bk;
            dv[k] = dd[u];
            xa[k] = L.w * dd[u] * bk;
            if (k < R.y) ti[k] = tt[u];
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < R.z; k += blockDim.x) {
        const T acc = tile_rowdot(val, lc, lrp, xa, k);
        xb[k] = xa[k] + L.w * dv[k] * (bp[k] - acc);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < R.y; k += blockDim.x) {
        const T rk = bp[k] - tile_rowdot(val, lc, lrp, xb, k);
        rr[k] = rk;
        ss[k] = ti[k] * rk;
    }
    for (int k = threadIdx.x; k < R.x; k += blockDim.x) {
        const int g = cell[k];
        L.y[g] = xb[k];  // the pre-smoothed iterate, read by k_tile_up
        L.bp[g] = bp[k];
    }
    __syncthreads();
    // four lanes per coarse cell, lane q takes child q; whole warps (shuffles)
    const int c0 = V.co_off[t];
    const int nco = V.co_off[t + 1] - c0;
    const int quads = (4 * nco + 31) & ~31;
    double part = 0;
    for (int gq = threadIdx.x; gq < quads; gq += blockDim.x) {
        const int J = gq >> 2, q = gq & 3;
        T acc = T(0);
        if (J < nco) {
            const int i = short4_at(V.ch[c0 + J], q);
            if (i >= 0) acc = rr[i] - L.tw * tile_rowdot(val, lc, lrp, ss, i);
        }
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        acc += __shfl_xor_sync(0xffffffffu, acc, 2);
        if (q == 0 && J < nco) {
            bc[V.co[c0 + J]] = acc;
            part += double(acc);
        }
    }
    if (coarse_sum) {
        if (publish_partial(part, partial, counter)) {
            const double s = fold_partials(partial, gridDim.x);
            if (threadIdx.x == 0) {
                *coarse_sum = s;
                *counter = 0;
            }
        }
    }
}

// xc: the coarse level's correction; mean_out (may be null): the volume mean
// of the result, folded by the last CTA, which then runs `epi`.
template <typename T, typename Epi, int NT>
__global__ void __launch_bounds__(NT)
    k_tile_up(LevelView<T> L, TileView<T> V, const T* __restrict__ xc, double* partial, unsigned* counter,
              double* mean_out, Epi epi) {
    pdl_entry();
    extern __shared__ __align__(16) unsigned char tile_smem[];
    T* e = reinterpret_cast<T*>(tile_smem);
    T* xp = e + V.n3max;
    T* dv = xp + V.n2max;
    T* ti = dv + V.n2max;
    T* bp = ti + V.n2max;
    T* xq = bp + V.n1max;
    T* val = xq + V.n1max;
    int* lrp = reinterpret_cast<int*>(val + V.emax);
    short* lc = reinterpret_cast<short*>(lrp + V.n2max + 1);
    const int t = blockIdx.x;
    const int4 R = V.ring[t];
    const int* cell = V.cell + V.cell_off[t];
    const int* own = V.own + V.cell_off[t];
    constexpr int CU = (kTileMaxCells + NT - 1) / NT;
    int g[CU], o[CU];
#pragma unroll
    for (int u = 0; u < CU; ++u) {
        const int k = threadIdx.x + u * NT;
        g[u] = k < R.w ? cell[k] : -1;
        o[u] = k < R.w ? own[k] : -1;
    }
    tile_stage_csr<T, NT>(V, t, R.z, val, lrp, lc);
    T ee[CU], yy[CU], dd[CU], tt[CU], bb[CU];
#pragma unroll
    for (int u = 0; u < CU; ++u) {
        const int k = threadIdx.x + u * NT;
        if (g[u] >= 0) {
            ee[u] = xc[o[u]];
            if (k < R.z) {
                yy[u] = L.y[g[u]];
                dd[u] = L.dinv[g[u]];
                tt[u] = L.tinv[g[u]];
            }
            if (k < R.y) bb[u] = L.bp[g[u]];
        }
    }
#pragma unroll
    for (int u = 0; u < CU; ++u) {
        const int k = threadIdx.x + u * NT;
        if (g[u] >= 0) {
            e[k] = ee[u];
            if (k < R.z) {
                xp[k] = yy[u];
                dv[k] = dd[u];
                ti[k] = tt[u];
            }
            if (k < R.y) bp[k] = bb[u];
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < R.z; k += blockDim.x) {
        const T ae = tile_rowdot(val, lc, lrp, e, k);
        xp[k] += e[k] - L.tw * ti[k] * ae;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < R.y; k += blockDim.x)
        xq[k] = xp[k] + L.w * dv[k] * (bp[k] - tile_rowdot(val, lc, lrp, xp, k));
    __syncthreads();
    double v = 0, w = 0;
    for (int k = threadIdx.x; k < R.x; k += blockDim.x) {
        const T out = xq[k] + L.w * dv[k] * (bp[k] - tile_rowdot(val, lc, lrp, xq, k));
        const int g = cell[k];
        L.x[g] = out;
        if (mean_out) {
            v += double(L.vol[g]) * double(out);
            if constexpr (Epi::kRz) w += epi.r[g] * double(out);
        }
    }
    if (mean_out) fold_mean(v, w, partial, counter, mean_out, L.cvol_inv, epi);
}

// tile copies of a level's CSR values: out[k] = val[pos[k]]
template <typename T>
__global__ void k_tile_gather(int m, const int* __restrict__ pos, const T* __restrict__ val, T* __restrict__ out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) out[k] = val[pos[k]];
}

// ---------------------------------------------------------------------------------
// The same two launches per level on constant-coefficient 16x16 levels (the
// levels of the vectorized kernels, stencil4.cuh: every block and its
// neighbours the same size, every coupling c0): the tile is the block plus a
// three-cell frame, a 22 x 22 square taken from the block and its eight
// neighbours (W, E, S, N from the neighbour table, the corners through them;
// cells of missing blocks -- walls -- do not exist), with no index lists.
// Each phase works on a square one cell smaller than the last.  The row
// arithmetic is that of the vectorized kernels (q_apply: the existing
// neighbours summed west, east, south, north).

namespace vt {
constexpr int R = 22;  // region side: 16 + 2 * 3
__device__ __forceinline__ int at(int i, int j) { return (j + 3) * R + (i + 3); }
}  // namespace vt

// the nine blocks around block b (index (by + 1) * 3 + (bx + 1), -1: none)
template <typename T>
__device__ __forceinline__ void vt_blocks(const SView<T>& L, int b, int* nb9) {
    if (threadIdx.x == 0) {
        const int4 c = *reinterpret_cast<const int4*>(L.nbr + 4 * b);
        const int4 none = make_int4(-1, -1, -1, -1);
        const int4 w = c.x >= 0 ? *reinterpret_cast<const int4*>(L.nbr + 4 * c.x) : none;
        const int4 e = c.y >= 0 ? *reinterpret_cast<const int4*>(L.nbr + 4 * c.y) : none;
        const int4 s = c.z >= 0 ? *reinterpret_cast<const int4*>(L.nbr + 4 * c.z) : none;
        const int4 n = c.w >= 0 ? *reinterpret_cast<const int4*>(L.nbr + 4 * c.w) : none;
        nb9[0] = c.x >= 0 ? w.z : s.x;  // south-west
        nb9[1] = c.z;
        nb9[2] = c.y >= 0 ? e.z : s.y;  // south-east
        nb9[3] = c.x;
        nb9[4] = b;
        nb9[5] = c.y;
        nb9[6] = c.x >= 0 ? w.w : n.x;  // north-west
        nb9[7] = c.w;
        nb9[8] = c.y >= 0 ? e.w : n.y;  // north-east
    }
}

// global cell of region cell (i, j), i, j in [-3, 18], or -1 when it does not exist
__device__ __forceinline__ int vt_cell(const int* nb9, int i, int j) {
    const int bx = i < 0 ? -1 : (i > 15 ? 1 : 0), by = j < 0 ? -1 : (j > 15 ? 1 : 0);
    const int B = nb9[(by + 1) * 3 + bx + 1];
    if (B < 0) return -1;
    return B * 256 + (j - 16 * by) * 16 + (i - 16 * bx);
}

// c0 (count * v - sum of the existing neighbours), neighbours in the order of q_apply
template <typename T>
__device__ __forceinline__ T vt_apply(const SView<T>& L, const T* v, const unsigned char* ex, int k) {
    T off = T(0);
    int cnt = 0;
    if (ex[k - 1]) off += v[k - 1], ++cnt;
    if (ex[k + 1]) off += v[k + 1], ++cnt;
    if (ex[k - vt::R]) off += v[k - vt::R], ++cnt;
    if (ex[k + vt::R]) off += v[k + vt::R], ++cnt;
    return L.c0 * (T(cnt) * v[k] - off);
}

template <typename T, typename TB>
__global__ void __launch_bounds__(kTileThreads)
    v_tile_down(SView<T> L, const TB* __restrict__ bin, const double* level_sum, T* __restrict__ bc, double* partial,
                unsigned* counter, double* coarse_sum) {
    pdl_entry();
    constexpr int N = vt::R * vt::R;
    __shared__ T sb[N], sd[N], sx[N], sy[N], sr[N], ss[N];
    __shared__ unsigned char ex[N];
    __shared__ int nb9[9];
    const int b = blockIdx.x;
    vt_blocks(L, b, nb9);
    const double mean = (L.singular && level_sum) ? *level_sum * L.cvol_inv : 0.0;
    __syncthreads();
    // the region's loads, all issued before any is used
    constexpr int QU = (N + kTileThreads - 1) / kTileThreads;
    int c[QU];
    TB a[QU];
    T vo[QU], dd[QU];
#pragma unroll
    for (int u = 0; u < QU; ++u) {
        const int q = threadIdx.x + u * kTileThreads;
        c[u] = q < N ? vt_cell(nb9, q % vt::R - 3, q / vt::R - 3) : -1;
    }
#pragma unroll
    for (int u = 0; u < QU; ++u) {
        if (c[u] >= 0) {
            a[u] = bin[c[u]];
            vo[u] = (mean != 0.0 && !L.const_vol) ? L.vol[c[u]] : L.vol0;
            dd[u] = L.dinv ? L.dinv[c[u]] : L.dinv0;
        }
    }
#pragma unroll
    for (int u = 0; u < QU; ++u) {
        const int q = threadIdx.x + u * kTileThreads;
        if (q >= N) continue;
        T bv = T(0), d = T(0);
        if (c[u] >= 0) {
            bv = mean != 0.0 ? T(double(a[u]) - double(vo[u]) * mean) : T(a[u]);
            d = dd[u];
        }
        ex[q] = c[u] >= 0;
        sb[q] = bv;
        sd[q] = d;
        sx[q] = L.w * d * bv;  // the first sweep from zero, pointwise
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 20 * 20; q += blockDim.x) {
        const int k = vt::at(q % 20 - 2, q / 20 - 2);
        if (ex[k]) sy[k] = sx[k] + L.w * sd[k] * (sb[k] - vt_apply(L, sx, ex, k));
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 18 * 18; q += blockDim.x) {
        const int k = vt::at(q % 18 - 1, q / 18 - 1);
        if (ex[k]) {
            const T r = sb[k] - vt_apply(L, sy, ex, k);
            sr[k] = r;
            ss[k] = sd[k] * r;
        }
    }
    __syncthreads();
    // t = r - wt A s on the block (into sx, no longer needed), and the block's
    // iterate (into L.y, read by v_tile_up) and projected right-hand side
    for (int q = threadIdx.x; q < 256; q += blockDim.x) {
        const int k = vt::at(q & 15, q >> 4);
        sx[k] = sr[k] - L.tw * vt_apply(L, ss, ex, k);
        L.y[b * 256 + q] = sy[k];
        L.bp[b * 256 + q] = sb[k];
    }
    __syncthreads();
    const int4 mp = *reinterpret_cast<const int4*>(L.map + 4 * b);
    double part = 0;
    if (mp.w == 1) {
        for (int q = threadIdx.x; q < 256; q += blockDim.x) {
            const int i = q & 15, j = q >> 4;
            const T t = sx[vt::at(i, j)];
            bc[mp.x * 256 + (mp.z + j) * 16 + mp.y + i] = t;
            part += double(t);
        }
    } else {
        // 2 x 2 aggregation in the order of v_restrict: row pairs, then the row above
        for (int q = threadIdx.x; q < 64; q += blockDim.x) {
            const int i = 2 * (q & 7), j = 2 * (q >> 3);
            const T h0 = sx[vt::at(i, j)] + sx[vt::at(i + 1, j)];
            const T d0 = sx[vt::at(i, j + 1)] + sx[vt::at(i + 1, j + 1)];
            const T t = h0 + d0;
            bc[mp.x * 256 + (mp.z + (j >> 1)) * 16 + mp.y + (i >> 1)] = t;
            part += double(t);
        }
    }
    if (coarse_sum) {
        if (publish_partial(part, partial, counter)) {
            const double s = fold_partials(partial, gridDim.x);
            if (threadIdx.x == 0) {
                *coarse_sum = s;
                *counter = 0;
            }
        }
    }
}

// e = P_tent x_c at the cell (li, lj) of block B (its map: coarse block, x / y offset, scale)
template <typename T>
__device__ __forceinline__ T vt_coarse(const SView<T>& L, const T* xc, int B, int li, int lj) {
    const int4 mp = *reinterpret_cast<const int4*>(L.map + 4 * B);
    if (mp.w == 1) return xc[mp.x * 256 + (mp.z + lj) * 16 + mp.y + li];
    return xc[mp.x * 256 + (mp.z + (lj >> 1)) * 16 + mp.y + (li >> 1)];
}

template <typename T, typename Epi>
__global__ void __launch_bounds__(kTileThreads)
    v_tile_up(SView<T> L, const T* __restrict__ xc, double* partial, unsigned* counter, double* mean_out, Epi epi) {
    pdl_entry();
    constexpr int N = vt::R * vt::R;
    __shared__ T se[N], sp[N], sq[N], sd[N], sb[N];
    __shared__ unsigned char ex[N];
    __shared__ int nb9[9];
    const int b = blockIdx.x;
    vt_blocks(L, b, nb9);
    __syncthreads();
    // the region's loads, all issued before any is used
    constexpr int QU = (N + kTileThreads - 1) / kTileThreads;
    int4 mp[QU];
    int c[QU], li[QU], lj[QU], ring[QU];
#pragma unroll
    for (int u = 0; u < QU; ++u) {
        const int q = threadIdx.x + u * kTileThreads;
        c[u] = -1;
        if (q < N) {
            const int i = q % vt::R - 3, j = q / vt::R - 3;
            const int bx = i < 0 ? -1 : (i > 15 ? 1 : 0), by = j < 0 ? -1 : (j > 15 ? 1 : 0);
            const int B = nb9[(by + 1) * 3 + bx + 1];
            li[u] = i - 16 * bx;
            lj[u] = j - 16 * by;
            // 3: the outer frame (e only), 2: x and D^-1 too, 1: also bp
            ring[u] = max(max(-i, i - 15), max(-j, j - 15));
            if (B >= 0) {
                c[u] = B * 256 + lj[u] * 16 + li[u];
                mp[u] = *reinterpret_cast<const int4*>(L.map + 4 * B);
            }
        }
    }
    T e[QU], x[QU], d[QU], bp[QU];
#pragma unroll
    for (int u = 0; u < QU; ++u) {
        e[u] = x[u] = d[u] = bp[u] = T(0);
        if (c[u] >= 0) {
            const int4 m = mp[u];
            e[u] = m.w == 1 ? xc[m.x * 256 + (m.z + lj[u]) * 16 + m.y + li[u]]
                            : xc[m.x * 256 + (m.z + (lj[u] >> 1)) * 16 + m.y + (li[u] >> 1)];
            if (ring[u] <= 2) {
                x[u] = L.y[c[u]];
                d[u] = L.dinv ? L.dinv[c[u]] : L.dinv0;
                if (ring[u] <= 1) bp[u] = L.bp[c[u]];
            }
        }
    }
#pragma unroll
    for (int u = 0; u < QU; ++u) {
        const int q = threadIdx.x + u * kTileThreads;
        if (q >= N) continue;
        ex[q] = c[u] >= 0;
        se[q] = e[u];
        sp[q] = x[u];
        sd[q] = d[u];
        sb[q] = bp[u];
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 20 * 20; q += blockDim.x) {
        const int k = vt::at(q % 20 - 2, q / 20 - 2);
        if (ex[k]) sp[k] += se[k] - L.tw * sd[k] * vt_apply(L, se, ex, k);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < 18 * 18; q += blockDim.x) {
        const int k = vt::at(q % 18 - 1, q / 18 - 1);
        if (ex[k]) sq[k] = sp[k] + L.w * sd[k] * (sb[k] - vt_apply(L, sp, ex, k));
    }
    __syncthreads();
    double v = 0, w = 0;
    for (int q = threadIdx.x; q < 256; q += blockDim.x) {
        const int k = vt::at(q & 15, q >> 4);
        const T o = sq[k] + L.w * sd[k] * (sb[k] - vt_apply(L, sq, ex, k));
        const int c = b * 256 + q;
        L.x[c] = o;
        if (mean_out) {
            v += (L.const_vol ? double(L.vol0) : double(L.vol[c])) * double(o);
            if constexpr (Epi::kRz) w += epi.r[c] * double(o);
        }
    }
    if (mean_out) fold_mean(v, w, partial, counter, mean_out, L.cvol_inv, epi);
}

}  // namespace tpa
