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

namespace tpa {

constexpr int kTileThreads = 256;

// One level's tiles in precision T (device pointers).
template <typename T>
struct TileView {
    int ntiles;
    int n3max, n2max, n1max;
    const int* cell;
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

template <typename T>
__host__ __device__ inline size_t tile_down_smem(int n3, int n2, int n1) {
    return sizeof(T) * (3 * size_t(n3) + size_t(n2) + 3 * size_t(n1)) + sizeof(int) * (size_t(n2) + 1);
}

template <typename T>
__host__ __device__ inline size_t tile_up_smem(int n3, int n2, int n1) {
    return sizeof(T) * (size_t(n3) + 3 * size_t(n2) + 2 * size_t(n1)) + sizeof(int) * (size_t(n2) + 1);
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
template <typename T, typename TB>
__global__ void __launch_bounds__(kTileThreads)
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
    int* lrp = reinterpret_cast<int*>(ss + V.n1max);
    const int t = blockIdx.x;
    const int4 R = V.ring[t];
    const int* cell = V.cell + V.cell_off[t];
    const int* rowp = V.lrp + V.lrp_off[t];
    const T* val = V.val + V.ent_off[t];
    const short* lc = V.lcol + V.ent_off[t];
    const double mean = (L.singular && level_sum) ? *level_sum * L.cvol_inv : 0.0;
    for (int k = threadIdx.x; k < R.w; k += blockDim.x) {
        const int g = cell[k];
        const T bk = proj_b<T, TB>(L, b, mean, g);
        const T dk = L.dinv[g];
        bp[k] = bk;
        dv[k] = dk;
        xa[k] = L.w * dk * bk;
        if (k < R.y) ti[k] = L.tinv[g];
    }
    for (int k = threadIdx.x; k <= R.z; k += blockDim.x) lrp[k] = rowp[k];
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
template <typename T, typename Epi>
__global__ void __launch_bounds__(kTileThreads)
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
    int* lrp = reinterpret_cast<int*>(xq + V.n1max);
    const int t = blockIdx.x;
    const int4 R = V.ring[t];
    const int* cell = V.cell + V.cell_off[t];
    const int* rowp = V.lrp + V.lrp_off[t];
    const T* val = V.val + V.ent_off[t];
    const short* lc = V.lcol + V.ent_off[t];
    for (int k = threadIdx.x; k < R.w; k += blockDim.x) {
        const int g = cell[k];
        e[k] = xc[L.owner[g]];
        if (k < R.z) {
            xp[k] = L.y[g];
            dv[k] = L.dinv[g];
            ti[k] = L.tinv[g];
        }
        if (k < R.y) bp[k] = L.bp[g];
    }
    for (int k = threadIdx.x; k <= R.z; k += blockDim.x) lrp[k] = rowp[k];
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

}  // namespace tpa
