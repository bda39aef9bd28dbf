// Block-structured level kernels: one CTA per nx x ny leaf block (or a capped
// grid that strides over blocks when the kernel also folds a reduction), one
// thread per cell, neighbours found by index arithmetic (inside the block, or
// in the same-size neighbour block across an edge); rows next to a coarse-fine
// edge use their exact assembled CSR row (see structure.cpp).  The block size
// is a template parameter (NXC = 16 for 16 x 16 blocks, 0 = read at run time),
// so the usual case indexes with shifts and masks.
//
// The phases are those of fused.cuh (the default V-cycle of
// src/solvers/multigrid/cycles.jl:46-77, ronaldremmerswaal/TwoPhaseAMR.jl):
// two pre-sweeps in one launch, residual, restriction P' r with the block map
// of the tentative transfer, prolongation P x_c, and the post-sweeps.
#pragma once

#include <cuda_runtime.h>

#include "fused.cuh"

namespace tpa {

template <typename T>
struct SView {
    int nx, ny, cpb, nblocks, n;
    const int* nbr;  // 4 per block (W, E, S, N) or -1
    const T* cx;     // east face coefficient per cell (null: constant c0)
    const T* cy;     // north face coefficient per cell
    T c0;
    const T* dinv;   // null: constant dinv0
    T dinv0;
    const int* ex;   // exception row per cell or -1 (null: none on this level)
    const int* ex_ptr;
    const int* ex_col;
    const T* ex_val;
    const int* map;  // 4 per block: coarse block, x offset, y offset, scale
    const T* vol;
    T vol0;          // every cell's volume when const_vol (the vectorized kernels skip the loads)
    int const_vol;
    T w, tw;
    int singular;
    double cvol_inv;
    T *b, *bp, *x, *y, *r, *s;
    int ccpb;        // cells per block on the coarser level (== cpb)
};

// compile-time block dimensions when NXC > 0
template <int NXC>
struct Blk {
    template <typename T>
    __device__ __forceinline__ static int nx(const SView<T>& L) { return NXC ? NXC : L.nx; }
    template <typename T>
    __device__ __forceinline__ static int ny(const SView<T>& L) { return NXC ? NXC : L.ny; }
    template <typename T>
    __device__ __forceinline__ static int cpb(const SView<T>& L) { return NXC ? NXC * NXC : L.cpb; }
};

template <typename T>
__device__ __forceinline__ T s_dinv(const SView<T>& L, int c) {
    return L.dinv ? L.dinv[c] : L.dinv0;
}

// Neighbour cell indices (W, E, S, N) of cell c = b * cpb + j * nx + i, -1 if none.
template <int NXC, typename T>
__device__ __forceinline__ void s_neighbours(const SView<T>& L, int b, int i, int j, int c, int nb[4]) {
    const int nx = Blk<NXC>::nx(L), ny = Blk<NXC>::ny(L), cpb = Blk<NXC>::cpb(L);
    nb[0] = i > 0 ? c - 1 : (L.nbr[4 * b] >= 0 ? L.nbr[4 * b] * cpb + j * nx + (nx - 1) : -1);
    nb[1] = i < nx - 1 ? c + 1 : (L.nbr[4 * b + 1] >= 0 ? L.nbr[4 * b + 1] * cpb + j * nx : -1);
    nb[2] = j > 0 ? c - nx : (L.nbr[4 * b + 2] >= 0 ? L.nbr[4 * b + 2] * cpb + (ny - 1) * nx + i : -1);
    nb[3] = j < ny - 1 ? c + nx : (L.nbr[4 * b + 3] >= 0 ? L.nbr[4 * b + 3] * cpb + i : -1);
}

// (A v)_c through a value functor f(q) (the stencil, or the exception row)
template <int NXC, typename T, typename F>
__device__ __forceinline__ T s_apply(const SView<T>& L, int b, int i, int j, int c, F f) {
    if (L.ex) {
        int e = L.ex[c];
        if (e >= 0) {
            T acc = T(0);
            for (int k = L.ex_ptr[e]; k < L.ex_ptr[e + 1]; ++k) acc += L.ex_val[k] * f(L.ex_col[k]);
            return acc;
        }
    }
    int nb[4];
    s_neighbours<NXC>(L, b, i, j, c, nb);
    T coef[4];
    if (L.cx) {
        coef[0] = nb[0] >= 0 ? L.cx[nb[0]] : T(0);
        coef[1] = nb[1] >= 0 ? L.cx[c] : T(0);
        coef[2] = nb[2] >= 0 ? L.cy[nb[2]] : T(0);
        coef[3] = nb[3] >= 0 ? L.cy[c] : T(0);
    } else {
#pragma unroll
        for (int d = 0; d < 4; ++d) coef[d] = nb[d] >= 0 ? L.c0 : T(0);
    }
    T diag = (coef[0] + coef[1]) + (coef[2] + coef[3]);
    T off = T(0);
#pragma unroll
    for (int d = 0; d < 4; ++d)
        if (nb[d] >= 0) off += coef[d] * f(nb[d]);
    return diag * f(c) - off;
}

// coarse cell that owns fine cell q (tentative transfer, block map)
template <int NXC, typename T>
__device__ __forceinline__ int s_owner(const SView<T>& L, int q) {
    const int nx = Blk<NXC>::nx(L), cpb = Blk<NXC>::cpb(L);
    int b = q / cpb, r = q - b * cpb;
    int i = r % nx, j = r / nx;
    const int* m = L.map + 4 * b;
    int sc = m[3];
    return m[0] * cpb + (m[2] + j / sc) * nx + (m[1] + i / sc);
}

#define TPA_S_CELL(bk)                                       \
    const int t = threadIdx.x;                               \
    const int i = t % Blk<NXC>::nx(L), j = t / Blk<NXC>::nx(L); \
    const int c = (bk) * Blk<NXC>::cpb(L) + t;

template <typename T, typename TB, int NXC>
__global__ void s_pre2(SView<T> L, const TB* __restrict__ bin, const double* level_sum) {
    pdl_entry();
    const int b = blockIdx.x;
    TPA_S_CELL(b);
    const double mean = (L.singular && level_sum) ? *level_sum * L.cvol_inv : 0.0;
    auto pb = [&](int q) {
        double v = double(bin[q]);
        if (L.singular) v -= double(L.vol[q]) * mean;
        return T(v);
    };
    auto x1 = [&](int q) { return L.w * s_dinv(L, q) * pb(q); };
    T bi = pb(c);
    T ax = s_apply<NXC>(L, b, i, j, c, x1);
    L.x[c] = x1(c) + L.w * s_dinv(L, c) * (bi - ax);
    L.bp[c] = bi;
}

template <typename T, int NXC>
__global__ void s_residual(SView<T> L) {
    pdl_entry();
    const int b = blockIdx.x;
    TPA_S_CELL(b);
    const T* x = L.x;
    T ri = L.bp[c] - s_apply<NXC>(L, b, i, j, c, [&](int q) { return x[q]; });
    L.r[c] = ri;
    L.s[c] = s_dinv(L, c) * ri;
}

// t = r - wt A s per fine cell, aggregated over the 2x2 (or 1x1) children into
// the coarse block quadrant; optional fold of the coarse RHS sum.  Strides over
// blocks so that the fold reads at most gridDim.x partials.
template <typename T, int NXC>
__global__ void s_restrict(SView<T> L, T* __restrict__ bc, double* partial, unsigned* counter, double* coarse_sum) {
    pdl_entry();
    extern __shared__ unsigned char smem_raw[];
    T* tile = reinterpret_cast<T*>(smem_raw);
    const T* sv = L.s;
    const int nx = Blk<NXC>::nx(L), ny = Blk<NXC>::ny(L), cpb = Blk<NXC>::cpb(L);
    double part = 0;
    for (int b = blockIdx.x; b < L.nblocks; b += gridDim.x) {
        TPA_S_CELL(b);
        __syncthreads();
        tile[t] = L.r[c] - L.tw * s_apply<NXC>(L, b, i, j, c, [&](int q) { return sv[q]; });
        __syncthreads();
        const int* m = L.map + 4 * b;
        const int cb = m[0], ox = m[1], oy = m[2], sc = m[3];
        if (sc == 1) {
            T v = tile[t];
            bc[cb * cpb + t] = v;
            part += double(v);
        } else if (i < nx / 2 && j < ny / 2) {
            const int f = 2 * j * nx + 2 * i;
            T v = tile[f] + tile[f + 1] + tile[f + nx] + tile[f + nx + 1];
            bc[cb * cpb + (oy + j) * nx + (ox + i)] = v;
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

// x += e - wt Dt^-1 A e with e = x_c[owner(.)], in place
template <typename T, int NXC>
__global__ void s_prolong(SView<T> L, const T* __restrict__ xc) {
    pdl_entry();
    const int b = blockIdx.x;
    TPA_S_CELL(b);
    auto e = [&](int q) { return xc[s_owner<NXC>(L, q)]; };
    T ae = s_apply<NXC>(L, b, i, j, c, e);
    L.x[c] += e(c) - L.tw * s_dinv(L, c) * ae;
}

template <typename T, int NXC>
__global__ void s_post1(SView<T> L) {
    pdl_entry();
    const int b = blockIdx.x;
    TPA_S_CELL(b);
    const T* x = L.x;
    L.y[c] = x[c] + L.w * s_dinv(L, c) * (L.bp[c] - s_apply<NXC>(L, b, i, j, c, [&](int q) { return x[q]; }));
}

template <typename T, int NXC, typename Epi = MeanOnly>
__global__ void s_post2(SView<T> L, double* partial, unsigned* counter, double* mean_out, Epi epi = Epi()) {
    pdl_entry();
    const T* y = L.y;
    double part = 0, rx = 0;
    for (int b = blockIdx.x; b < L.nblocks; b += gridDim.x) {
        TPA_S_CELL(b);
        T v = y[c] + L.w * s_dinv(L, c) * (L.bp[c] - s_apply<NXC>(L, b, i, j, c, [&](int q) { return y[q]; }));
        L.x[c] = v;
        part += double(L.vol[c]) * double(v);
        if constexpr (Epi::kRz) rx += epi.r[c] * double(v);
    }
    if (mean_out) fold_mean(part, rx, partial, counter, mean_out, L.cvol_inv, epi);
}

// y = A x on the finest level with the partial x'y, folded by `fold(sum)` in the
// last block (CG operator product)
template <typename T, int NXC, typename Fold>
__device__ __forceinline__ void s_apply_dot(const SView<T>& L, const T* x, T* y, double* partial, unsigned* counter,
                                            Fold fold) {
    double part = 0;
    for (int b = blockIdx.x; b < L.nblocks; b += gridDim.x) {
        TPA_S_CELL(b);
        T v = s_apply<NXC>(L, b, i, j, c, [&](int q) { return x[q]; });
        y[c] = v;
        part += double(x[c]) * double(v);
    }
    if (publish_partial(part, partial, counter)) {
        double s = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            fold(s);
            *counter = 0;
        }
    }
}

// s_apply_dot with the operand formed where it is read: ld(q) = x_q, and
// keep(c, x_c) stores the operand of the CTA's own cells; y has the storage
// type P of the product
template <typename T, int NXC, typename Ld, typename Keep, typename P, typename Fold>
__device__ __forceinline__ void s_apply_dot_ld(const SView<T>& L, Ld ld, Keep keep, P* y, double* partial,
                                               unsigned* counter, Fold fold) {
    double part = 0;
    for (int b = blockIdx.x; b < L.nblocks; b += gridDim.x) {
        TPA_S_CELL(b);
        const T v = s_apply<NXC>(L, b, i, j, c, ld);
        const T xc = ld(c);
        keep(c, xc);
        y[c] = P(v);
        part += double(xc) * double(v);
    }
    if (publish_partial(part, partial, counter)) {
        double s = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            fold(s);
            *counter = 0;
        }
    }
}

#undef TPA_S_CELL

}  // namespace tpa
