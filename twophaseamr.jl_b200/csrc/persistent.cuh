// One V-cycle in one cooperative launch (CSR levels): the phases of the fused
// cycle (fused.cuh; src/solvers/multigrid/cycles.jl:46-77 of
// ronaldremmerswaal/TwoPhaseAMR.jl) separated by grid-wide barriers instead of
// kernel boundaries, with one CTA of 1024 threads per SM.  The coarse tail runs
// in CTA 0 while the others wait at the next barrier.
//
// The barrier is bounded: a CTA that polls more than `spins` times (a launch
// parameter, kBarrierSpins by default) records err = 1 and goes on, and every
// later barrier returns at once once err is set, so a fault in the barrier
// protocol ends the launch with an error status instead of a hang.  A
// cooperative launch guarantees that every CTA is resident, so in correct
// operation no wait is long; a limit of 0 gives up at the first unsuccessful
// poll (the failure path, exercised by the tests).
#pragma once

#include <cuda_runtime.h>

#include "fused.cuh"

namespace tpa {

constexpr unsigned long long kBarrierSpins = 1ull << 24;  // x >= 32 ns: about half a second

// bar[0]: arrivals, bar[1]: generation.  With `partial`, every CTA also
// publishes the block sum of v, and the last CTA to arrive folds them in block
// order into *out (times `scale`) before it releases the others.
__device__ __forceinline__ void grid_barrier(unsigned* bar, int* err, unsigned long long spin_limit, double v = 0.0,
                                             double* partial = nullptr, double* out = nullptr, double scale = 1.0) {
    __shared__ bool last;
    const bool fold = partial != nullptr;
    double b = 0;
    if (fold) b = block_sum_all(v);
    __syncthreads();
    volatile unsigned* gen = bar + 1;
    unsigned g = 0;
    if (threadIdx.x == 0) {
        g = *gen;
        if (fold) partial[blockIdx.x] = b;
        __threadfence();
        last = atomicAdd(bar, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last) {
        if (fold) {
            __threadfence();
            const double s = fold_partials(partial, gridDim.x);
            if (threadIdx.x == 0 && out) *out = s * scale;
        }
        if (threadIdx.x == 0) {
            bar[0] = 0;
            __threadfence();
            atomicAdd(const_cast<unsigned*>(gen), 1u);
        }
    } else if (threadIdx.x == 0) {
        unsigned long long spins = 0;
        while (*gen == g) {
            if (*(volatile int*)err) break;
            if (++spins > spin_limit) {
                atomicExch(err, 1);
                break;
            }
            __nanosleep(32);
        }
    }
    if (threadIdx.x == 0) __threadfence();
    __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(kTailThreads, 1)
    k_vcycle_grid(const LevelView<T>* __restrict__ levels, int t, int nl, const double* __restrict__ r,
                  const double* rsum, double* mean_out, const double* __restrict__ G, int gn, double* partial,
                  unsigned* bar, double* lsum, int* err, unsigned long long spins) {
    pdl_entry();
    const int gt = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
    for (int l = 0; l < t; ++l) {
        const LevelView<T> L = levels[l];
        double mean = 0;
        if (L.singular) mean = (l == 0 ? *rsum : __ldcg(lsum + l)) * L.cvol_inv;
        if (l == 0)
            for (int i = gt; i < L.n; i += gs) pre2_cell<T, double>(L, r, mean, i);
        else
            for (int i = gt; i < L.n; i += gs) pre2_cell<T, T>(L, L.b, mean, i);
        grid_barrier(bar, err, spins);
        for (int i = gt; i < L.n; i += gs) residual_cell(L, i);
        grid_barrier(bar, err, spins);
        T* bc = levels[l + 1].b;
        const int quads = (4 * L.nc + 31) & ~31;
        double part = 0;
        for (int g = gt; g < quads; g += gs) {
            const T v = restrict_quad(L, g >> 2, g & 3);
            if ((g & 3) == 0 && (g >> 2) < L.nc) {
                bc[g >> 2] = v;
                part += double(v);
            }
        }
        const bool next_sum = l + 1 < t && levels[l + 1].singular;
        grid_barrier(bar, err, spins, part, partial, next_sum ? lsum + l + 1 : nullptr);
    }
    if (blockIdx.x == 0)
        tail_run<T, double>(levels, t, nl, t == 0 ? r : nullptr, G, gn,
                            t == 0 && levels[0].singular ? mean_out : nullptr);
    grid_barrier(bar, err, spins);
    for (int l = t - 1; l >= 0; --l) {
        const LevelView<T> L = levels[l];
        const T* xc = levels[l + 1].x;
        for (int i = gt; i < L.n; i += gs) prolong_cell(L, xc, i);
        grid_barrier(bar, err, spins);
        for (int i = gt; i < L.n; i += gs) sweep_cell(L, L.x, L.y, i);
        grid_barrier(bar, err, spins);
        const bool want_mean = l == 0 && L.singular;
        double part = 0;
        for (int i = gt; i < L.n; i += gs) {
            sweep_cell(L, L.y, L.x, i);
            if (want_mean) part += double(L.vol[i]) * double(L.x[i]);
        }
        if (want_mean) grid_barrier(bar, err, spins, part, partial, mean_out, L.cvol_inv);
        else grid_barrier(bar, err, spins);
    }
}

}  // namespace tpa
