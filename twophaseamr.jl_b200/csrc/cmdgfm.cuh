// The CMDGFM two-block solve on the device (cmdgfm.cu): residual replacement
// around scaled BiCGSTAB runs with the block-lower preconditioner, the
// context's tree GMG V-cycle on the reduced pressure block and the incomplete
// LU of the jump block's local Schur complement.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "cmdgfm.hpp"
#include "device.cuh"

namespace tpa {

// The system as the C-ABI takes it (host arrays, 0-based).
struct CmdgfmInput {
    CsrRows m;                        // n x n, rows: np pressures, then nx jumps
    int64_t np = 0;
    std::vector<double> rhs;          // n
    std::vector<int32_t> cell, anchor;  // np: cell and anchor cell of each pressure unknown
    std::vector<double> weight;       // n: defect weight
    CsrRows extra;                    // na x n: the omitted anchor rows
    std::vector<double> extra_rhs, extra_weight;
    std::vector<double> row_scale, col_scale;  // n
    double tolerance = 1.4901161193847656e-08;
    int max_iterations = 500;
    int precision = 0;                // V-cycle: 0 FP64, 1 FP32
    bool warm_start = false;          // `_cmdgfm_initial_solution!` before the loop
    std::vector<double> initial;      // np: the previous increment, reduced (may be empty)
};

struct CmdgfmStats {
    bool converged = false;
    int iterations = 0, attempts = 0;
    double initial_residual = 0, final_residual = 0;
    double pressure_defect = 0, jump_defect = 0, anchor_defect = 0;
    double device_ms = 0;
    int launches = 0;
    bool inverse = false;  // the jump block went through the factors' inverses
    bool initial_guess_used = false;
};

// a triangular factor laid out for its solve on the device (cmdgfm.cu)
struct TriView {
    int nlev, nnz, seq;
    const int32_t* lev;
    const int32_t* rows;
    const int32_t* ptr;
    const int32_t* col;
    const double* val;
    const double* inv;
};

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        if (count <= n && p) return;
        if (p) cudaFree(p);
        p = nullptr;
        n = count;
        if (count) TPA_CUDA(cudaMalloc(&p, count * sizeof(T)));
    }
    void upload(const T* h, size_t count, cudaStream_t s) {
        alloc(std::max<size_t>(count, 1));
        if (count) TPA_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

class CmdgfmDevice {
public:
    CmdgfmDevice() = default;
    CmdgfmDevice(const CmdgfmDevice&) = delete;
    CmdgfmDevice& operator=(const CmdgfmDevice&) = delete;
    ~CmdgfmDevice() {
        for (auto& g : exec_)
            if (g) cudaGraphExecDestroy(g);
    }
    // Solves in place of `_project_cmdgfm_assembled!`'s linear part; the
    // solution (n) is a host array.  `ds` carries the pressure hierarchy.
    void solve(DeviceSolver& ds, const CmdgfmInput& in, const CmdgfmFactor& f, double* solution, CmdgfmStats& st);

private:
    // one BiCGSTAB run on b (device): returns iterations; x holds the result
    int bicgstab(DeviceSolver& ds, const CmdgfmInput& in, const CmdgfmFactor& f, bool preconditioned, double rtol,
                 int itmax, cudaStream_t s);
    void precondition(DeviceSolver& ds, const CmdgfmFactor& f, const double* src, double* dst, int precision,
                      cudaStream_t s);
    void spmv(const double* x, double* y, int mode, cudaStream_t s);
    void jump_apply(const double* src, const double* rows, const double* cols, const double* zp, double* dst,
                    cudaStream_t s);
    DevBuf<double> ones_;
    void enqueue_iteration(DeviceSolver& ds, const CmdgfmFactor& f, bool preconditioned, int precision,
                           cudaStream_t s, cudaGraphConditionalHandle handle, int set_cond);
    cudaGraphExec_t loop_graph(DeviceSolver& ds, const CmdgfmFactor& f, bool preconditioned, int precision,
                               cudaStream_t s);
    // captured BiCGSTAB loops (without / with the preconditioner) and what they captured
    cudaGraphExec_t exec_[2] = {nullptr, nullptr};
    std::vector<uintptr_t> key_[2];
    int body_launches_[2] = {0, 0};
    int64_t n_ = 0, np_ = 0, nx_ = 0, na_ = 0, ncells_ = 0;
    int launches_ = 0;
    int precision_ = 0;
    // system
    DevBuf<int64_t> mptr_, eptr_;
    DevBuf<int32_t> mcol_, ecol_, cell_, anchor_, gptr_, gidx_, ganchor_;
    DevBuf<double> mval_, eval_, rhs_, weight_, erhs_, eweight_, rows_, cols_;
    int ngroups_ = 0, anchor1_ = -1;
    DevBuf<unsigned> counter_;  // fold counter of the scatter (reset by its last block)
    // jump block: C, and the factors in the order of their level schedules
    DevBuf<int64_t> cptr_;
    DevBuf<int32_t> ccol_, lptr_, lcol_, uptr_, ucol_, lrows_, lsched_, urows_, usched_;
    DevBuf<double> cval_, lval_, uval_, piv_;
    int llevels_ = 0, ulevels_ = 0, jstaged_ = 0;
    size_t jsmem_ = 0;
    TriView lview_{}, uview_{};
    // the factors' inverses by rows (used when `inverse_`)
    bool inverse_ = false;
    DevBuf<int64_t> liptr_, uiptr_;
    DevBuf<int32_t> licol_, uicol_;
    DevBuf<double> lival_, uival_;
    // vectors
    DevBuf<double> sol_, corr_, x_, r_, c_, p_, v_, s_, t_, y_, z_, full_, zfull_, zp_, jr_, partial_;
    DevBuf<double> state_;
};

}  // namespace tpa
