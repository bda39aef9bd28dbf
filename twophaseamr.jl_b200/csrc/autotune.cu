// Layout autotuner of the device V-cycle: the reference has no counterpart
// (its cycle runs on the host, src/solvers/multigrid/cycles.jl:46-77 of
// ronaldremmerswaal/TwoPhaseAMR.jl).  Which levels run in the coarse tail and
// in how many CTAs, which levels use the stencil (block-structured) kernels and
// their vectorized form, and programmatic dependent launch are timed on the
// hierarchy at hand; the configurations differ only in data movement, so every
// candidate gives the same V-cycle to rounding.
#include <cmath>

#include "device.cuh"

namespace tpa {
namespace {

__global__ void k_pattern(int n, const double* __restrict__ vol, double* __restrict__ r) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = vol[i] * sin(0.37 * double(i) + 0.1);
}

}  // namespace

void DeviceSolver::reconfigure(const Hierarchy& h, const TuneConfig& c) {
    TPA_CUDA(cudaSetDevice(device_));
    TPA_CUDA(cudaStreamSynchronize(stream_));
    tune_ = c;
    build_views();
    upload_structured(h);
    upload_tiles(h);
}

double DeviceSolver::time_vcycles(int precision, int count) {
    TPA_CUDA(cudaSetDevice(device_));
    if (count <= 0) throw Error(1, "count must be positive");
    const int n = levels_[0].n;
    k_pattern<<<(n + kThreads - 1) / kThreads, kThreads, 0, stream_>>>(n, levels_[0].d.vol.p, tmp_.p);
    // warm-up (and lazy set-up), then the timed cycles
    vcycle(tmp_.p, z_.p, precision);
    vcycle(tmp_.p, z_.p, precision);
    cudaEvent_t e0, e1;
    TPA_CUDA(cudaEventCreate(&e0));
    TPA_CUDA(cudaEventCreate(&e1));
    TPA_CUDA(cudaEventRecord(e0, stream_));
    for (int k = 0; k < count; ++k) vcycle(tmp_.p, z_.p, precision);
    TPA_CUDA(cudaEventRecord(e1, stream_));
    TPA_CUDA(cudaEventSynchronize(e1));
    TPA_CUDA(cudaGetLastError());
    check_barrier();
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return double(ms) / count;
}

}  // namespace tpa
