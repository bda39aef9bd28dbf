// The coarse tail with its levels staged in shared memory.
//
// `k_tail` (fused.cuh) runs the levels of at most a few thousand cells and the
// dense coarse solve in one CTA; every phase of it walks CSR rows, so on the
// global-memory copy each phase waits on chains of L2 loads.  `k_tail_smem`
// copies each tail level's operator, diagonals, volumes, transfer lists and
// work vectors into shared memory once per V-cycle (batched loads), points a
// shared copy of the level views at them, runs the same phases (`tail_run`,
// so the arithmetic and the results are those of `k_tail`), and writes back
// the one vector read after it: the correction of its first level.  The dense
// coarse inverse stays in global memory.
#pragma once

#include <cuda_runtime.h>

#include "fused.cuh"

namespace tpa {

constexpr int kTailSmemMaxLevels = 32;

__host__ __device__ inline size_t tail_align16(size_t b) { return (b + 15) & ~size_t(15); }

// Shared-memory bytes of one staged tail level (n cells, nnz entries, nc cells
// on the next level; `last`: the coarsest level, which has no transfer).
template <typename T>
__host__ __device__ inline size_t tail_level_bytes(int n, int nnz, int nc, bool last) {
    // T: val (nnz), dinv, vol, x, y, b, bp, r, s (n each), tinv (n, not last)
    const size_t tb = sizeof(T) * (size_t(nnz) + size_t(n) * (last ? 8 : 9));
    // int: rp (n + 1), ci (nnz), owner, child (n each) and cptr (nc + 1), not last
    const size_t ib = sizeof(int) * (size_t(n) + 1 + size_t(nnz) + (last ? 0 : 2 * size_t(n) + size_t(nc) + 1));
    return tail_align16(tb) + tail_align16(ib);
}

// copy n values, up to 8 loads in flight per thread
template <typename V>
__device__ __forceinline__ void tail_stage(V* dst, const V* src, int n) {
    constexpr int U = 8;
    for (int base = threadIdx.x; base < n; base += U * blockDim.x) {
        V v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = base + u * blockDim.x;
            if (i < n) v[u] = src[i];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = base + u * blockDim.x;
            if (i < n) dst[i] = v[u];
        }
    }
}

// One CTA, no cluster.  `gl`: the level views in global memory.
template <typename T, typename TB>
__global__ void __launch_bounds__(kTailThreads)
    k_tail_smem(const LevelView<T>* __restrict__ gl, int first, int nl, const TB* top_b,
                const double* __restrict__ G, int gn, double* mean_out) {
    pdl_entry();
    extern __shared__ __align__(16) unsigned char tail_smem[];
    __shared__ LevelView<T> lv[kTailSmemMaxLevels];
    if (threadIdx.x == 0) {
        size_t off = 0;
        for (int l = 0; l < nl; ++l) {
            LevelView<T> v = gl[l];
            if (l >= first) {
                const bool last = l == nl - 1;
                const int n = v.n, nnz = v.rp[n], nc = last ? 0 : v.nc;
                T* t = reinterpret_cast<T*>(tail_smem + off);
                v.val = t;
                t += nnz;
                v.dinv = t;
                t += n;
                v.vol = t;
                t += n;
                v.x = t;
                t += n;
                v.y = t;
                t += n;
                v.b = t;
                t += n;
                v.bp = t;
                t += n;
                v.r = t;
                t += n;
                v.s = t;
                t += n;
                if (!last) {
                    v.tinv = t;
                    t += n;
                }
                int* q = reinterpret_cast<int*>(tail_smem + off +
                                                tail_align16(sizeof(T) * (size_t(nnz) + size_t(n) * (last ? 8 : 9))));
                v.rp = q;
                q += n + 1;
                v.ci = q;
                q += nnz;
                if (!last) {
                    v.owner = q;
                    q += n;
                    v.child = q;
                    q += n;
                    v.cptr = q;
                }
                off += tail_level_bytes<T>(n, nnz, nc, last);
            }
            lv[l] = v;
        }
    }
    __syncthreads();
    for (int l = first; l < nl; ++l) {
        const LevelView<T>& g = gl[l];
        const LevelView<T>& s = lv[l];
        const bool last = l == nl - 1;
        const int n = s.n;
        tail_stage(const_cast<int*>(s.rp), g.rp, n + 1);
        const int m = __ldg(g.rp + n);
        tail_stage(const_cast<int*>(s.ci), g.ci, m);
        tail_stage(const_cast<T*>(s.val), g.val, m);
        tail_stage(const_cast<T*>(s.dinv), g.dinv, n);
        tail_stage(const_cast<T*>(s.vol), g.vol, n);
        if (!last) {
            tail_stage(const_cast<T*>(s.tinv), g.tinv, n);
            tail_stage(const_cast<int*>(s.owner), g.owner, n);
            tail_stage(const_cast<int*>(s.child), g.child, n);
            tail_stage(const_cast<int*>(s.cptr), g.cptr, s.nc + 1);
        }
        // the first level's right-hand side comes from the kernel before
        if (l == first && first > 0) tail_stage(s.b, g.b, n);
    }
    __syncthreads();
    tail_run<T, TB>(lv, first, nl, top_b, G, gn, mean_out);
    __syncthreads();
    // the correction of the first tail level, read by the level above
    tail_stage(gl[first].x, lv[first].x, lv[first].n);
}

}  // namespace tpa
