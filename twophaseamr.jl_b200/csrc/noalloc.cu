// Residual norms without any device allocation.
//
// Some callers cannot call cudaMalloc: callers whose device memory is owned by
// a pool or arena they must not bypass, and embedded hosts that forbid runtime
// allocation.  `tpa_residual_norms_noalloc` gives them the two norms of
// `_integrated_residual_norms` (src/solvers/multigrid/cycles.jl:210-221 in
// ronaldremmerswaal/TwoPhaseAMR.jl) with all scratch in one file-scope
// `__device__` array of fixed size (kNoAllocBlocks partial sums per norm, about
// 14 KiB), which every GPU that loads this library holds until the process
// exits.  No tpa_context state is used, so no hierarchy upload is triggered.
//
// Per call, on the legacy default stream: the fold counter is cleared with
// cudaMemsetAsync (so a launch that was aborted, or two calls that overlapped,
// cannot leave it nonzero for the next call), the kernel runs, and a
// synchronous cudaMemcpy returns the two norms.
#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/tpagmg.h"
#include "fused.cuh"

namespace {

constexpr int kNoAllocBlocks = 592;  // fixed grid: 4 CTAs per SM on 148 SMs
constexpr int kNoAllocThreads = 256;
constexpr int kMaxDevices = 64;

struct NormsScratch {
    double l2[kNoAllocBlocks];
    double vol[kNoAllocBlocks];
    double mx[kNoAllocBlocks];
    double result[2];
    unsigned counter;  // blocks done; cleared by the host before every launch
};

// The scratch of every call on this device.  In host code this name is only a
// host-side stand-in: its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) NormsScratch g_norms_scratch;

__global__ void __launch_bounds__(kNoAllocThreads)
    k_norms_noalloc(const double* __restrict__ r, const double* __restrict__ vol, int64_t n, NormsScratch* S) {
    __shared__ double sa[32], sv[32], sm[32];
    __shared__ int nan_seen;
    __shared__ bool last;
    double a = 0, v = 0, m = 0;
    bool nan = false;
    // 64-bit index: the grid stride must not overflow for n near the maximum
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double V = vol[i];
        if (!(V > 0)) continue;
        const double s = r[i] / V;
        a += V * s * s;
        v += V;
        const double q = fabs(r[i]) / V;
        if (q != q) nan = true;
        m = fmax(m, q);
    }
    if (threadIdx.x == 0) nan_seen = 0;
    __syncthreads();
    if (nan) nan_seen = 1;
    for (int o = 16; o; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        v += __shfl_down_sync(0xffffffffu, v, o);
        m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (!lane) {
        sa[wid] = a;
        sv[wid] = v;
        sm[wid] = m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ba = 0, bv = 0, bm = 0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) {
            ba += sa[w];
            bv += sv[w];
            bm = fmax(bm, sm[w]);
        }
        S->l2[blockIdx.x] = ba;
        S->vol[blockIdx.x] = bv;
        S->mx[blockIdx.x] = nan_seen ? NAN : bm;
        __threadfence();
        last = atomicAdd(&S->counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    // the last block folds the partials in block order (same result every call)
    double fa = tpa::fold_partials(S->l2, gridDim.x);
    double fv = tpa::fold_partials(S->vol, gridDim.x);
    double fm = tpa::fold_partials_max(S->mx, gridDim.x);
    if (threadIdx.x == 0) {
        S->result[0] = sqrt(fa / fv);
        S->result[1] = fm;
    }
}

std::mutex g_setup_mutex;
NormsScratch* g_scratch_ptr[kMaxDevices] = {};

}  // namespace

namespace tpa {
void set_context_error(tpa_context* ctx, const std::string& msg);  // api.cpp
}

namespace {
void set_error(tpa_context* ctx, const std::string& msg) {
    if (ctx) tpa::set_context_error(ctx, msg);
}
}  // namespace

extern "C" tpa_status tpa_residual_norms_noalloc(tpa_context* ctx, const double* r, const double* volumes, int64_t n,
                                                 double out[2]) {
    if (!r || !volumes || !out) {
        set_error(ctx, "tpa_residual_norms_noalloc: null residual, volumes or output");
        return TPA_ERR_INVALID_ARG;
    }
    if (n < 1 || n > int64_t(INT32_MAX)) {
        set_error(ctx, "tpa_residual_norms_noalloc: n must lie in [1, 2147483647] (32-bit cell indices); got " +
                           std::to_string(n));
        return TPA_ERR_INVALID_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_error(ctx, std::string("tpa_residual_norms_noalloc: no current CUDA device: ") + cudaGetErrorString(e));
        return TPA_ERR_CUDA;
    }
    NormsScratch* S = nullptr;
    {
        // Set-up, once per device with that device current: the device address
        // of the static scratch (the host-side name is only a stand-in).  The
        // cached address belongs to this process's context on the device; it
        // does not survive cudaDeviceReset.
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_norms_scratch);
            if (e != cudaSuccess || !p) {
                set_error(ctx, std::string("tpa_residual_norms_noalloc: cudaGetSymbolAddress failed: ") +
                                   cudaGetErrorString(e));
                return TPA_ERR_CUDA;
            }
            g_scratch_ptr[dev] = static_cast<NormsScratch*>(p);
        }
        S = g_scratch_ptr[dev];
    }
    // the last-block fold needs a zero counter: cleared before every launch
    e = cudaMemsetAsync(reinterpret_cast<char*>(S) + offsetof(NormsScratch, counter), 0, sizeof(unsigned), 0);
    if (e == cudaSuccess) {
        k_norms_noalloc<<<kNoAllocBlocks, kNoAllocThreads>>>(r, volumes, n, S);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(out, reinterpret_cast<const char*>(S) + offsetof(NormsScratch, result), 2 * sizeof(double),
                       cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        set_error(ctx, std::string("tpa_residual_norms_noalloc: ") + cudaGetErrorString(e));
        return TPA_ERR_CUDA;
    }
    return TPA_OK;
}
