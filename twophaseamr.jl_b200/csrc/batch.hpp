// Merged batch of independent pressure solves on one GPU (see batch.cuh).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "batch.cuh"
#include "device.cuh"

namespace tpa {

class BatchSolver {
public:
    // Builds the batch levels from the problems' host hierarchies and uploads
    // them; the hierarchies are not referenced afterwards.
    BatchSolver(int device, const std::vector<const Hierarchy*>& hierarchies);
    ~BatchSolver();
    BatchSolver(const BatchSolver&) = delete;
    BatchSolver& operator=(const BatchSolver&) = delete;

    int count() const { return K_; }
    int64_t fine_cells() const { return nfine_; }
    // fine-space offset of every problem (count + 1 entries)
    const std::vector<int64_t>& offsets() const { return F_; }
    int levels() const { return L_; }
    int tail_levels() const { return T_; }
    int64_t level_rows(int j) const { return lev_[size_t(j)].n; }
    cudaStream_t stream() const { return stream_; }
    void set_stream(cudaStream_t s) { stream_ = s ? s : own_stream_; }
    int kernel_launches() const { return launches_; }
    void reset_launches() { launches_ = 0; }
    float last_ms() const { return last_ms_; }

    // `solve!` of every problem: rhs (strong form) and x (initial guess in,
    // solution out) are device arrays of the concatenated fine cells (problem
    // order).  status[k] != 0 marks a problem rejected before its solve
    // (messages[k] says why).
    void solve(const double* rhs, double* x, double rtol, double atol, int max_cycles, int compatibility,
               int precision, std::vector<SolveStats>& stats, std::vector<int>& status,
               std::vector<std::string>& messages);

private:
    struct BLevelHost {
        int n = 0, nitems = 0;
        DevArray<int> rp, ci, owner, cptr, child, pfirst, pcount;
        DevArray<BItem> items;
        DevArray<double> cvol_inv, lsum;
        DevArray<double> val_d, wd_d, td_d, vol_d, b_d, bp_d, x_d, y_d, r_d, s_d;
        DevArray<float> val_f, wd_f, td_f, vol_f, b_f, bp_f, x_f, y_f, r_f, s_f;
    };

    void build(const std::vector<const Hierarchy*>& hierarchies);
    template <typename T> void enqueue_vcycle(const double* r);
    void enqueue_z(int precision, int init);
    void enqueue_body(int precision, cudaGraphConditionalHandle handle, bool in_graph);
    cudaGraphExec_t graph(int precision);
    double total_volume(int k) const;

    int device_;
    cudaStream_t stream_ = nullptr, own_stream_ = nullptr;
    int K_ = 0, L_ = 0, T_ = 1, nfi_ = 0;
    int64_t nfine_ = 0;
    std::vector<int64_t> F_;
    std::vector<double> comp_vol_, total_vol_;
    std::vector<BLevelHost> lev_;
    std::vector<BLevel<double>> vd_;
    std::vector<BLevel<float>> vf_;
    DevArray<BLevel<double>> vd_dev_;
    DevArray<BLevel<float>> vf_dev_;
    DevArray<BTail> tails_;
    DevArray<double> G_;
    DevArray<BFItem> fitems_;
    DevArray<int> fpfirst_, fpcount_, frp_, fci_;
    DevArray<double> fval_, fvol_;
    DevArray<double> b_, x_, r_, p_, ap_, z_, rhs_, x0_, partial_, partial2_, mean_, kvec_;
    DevArray<unsigned> counters_;
    DevArray<BState> state_;
    DevArray<int> active_, kint_;
    cudaGraphExec_t exec_[2] = {nullptr, nullptr};
    int body_launches_[2] = {0, 0};
    int launches_ = 0;
    float last_ms_ = 0;
};

}  // namespace tpa
