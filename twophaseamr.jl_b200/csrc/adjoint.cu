// Adjoint of the pressure solve: the face-coefficient gradient kernel.
//
// The solve maps a strong right-hand side f and face coefficients kappa to
//   p = G S(kappa)^+ Pi (V f),   S = J' sqrt(k) K sqrt(k) J,
// with Pi the component projection of the integrated right-hand side and G the
// volume-mean gauge (solvers/multigrid/elliptic_solver.jl:628-675, 132-190 of
// ronaldremmerswaal/TwoPhaseAMR.jl; operator src/operators/elliptic.jl:157-257,
// 1125-1180).  Because S is symmetric and Pi' = G, the adjoint state of a loss
// with dJ/dp = pbar is lam = G S^+ Pi pbar, i.e. the same solve with strong
// right-hand side pbar / V; then dJ/df = V lam, and
//   dJ/dkappa_f = -lam' (dS/dkappa_f) p
//               = -[w_f (K sqrt(k) u)_f + u_f (K sqrt(k) w)_f] / (2 sqrt(k_f)),
// u = J p, w = J lam (area-weighted face jumps).  On a diagonal row of K this is
// -K_ff u_f w_f.  The preconditioner does not enter: the gradient is that of the
// converged solve, so no V-cycle iterate is stored.
#include <cmath>

#include "device.cuh"

namespace tpa {

namespace {

// One thread per face.  The row of K is short (1 on conforming faces, a vertex
// patch at hanging vertices); the neighbour jumps are recomputed from p and lam
// rather than stored.
__global__ void k_face_gradient(int nf, const int* __restrict__ fm, const int* __restrict__ fp,
                                const double* __restrict__ area, const int* __restrict__ kptr,
                                const int* __restrict__ kcol, const double* __restrict__ kval,
                                const double* __restrict__ sk, const double* __restrict__ p,
                                const double* __restrict__ lam, double* __restrict__ g) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
        const int m = fm[f], q = fp[f];
        const double af = area[f];
        const double uf = af * (p[q] - p[m]);
        const double wf = af * (lam[q] - lam[m]);
        const double sf = sk[f];
        // diagonal entry first: its sqrt(k_f) cancels exactly
        int k = kptr[f];
        const double kd = kval[k];
        double acc = 2.0 * kd * uf * wf;
        double U = 0.0, W = 0.0;
        for (++k; k < kptr[f + 1]; ++k) {
            const int h = kcol[k];
            const double ah = area[h];
            const double c = kval[k] * sk[h];
            U += c * ah * (p[fp[h]] - p[fm[h]]);
            W += c * ah * (lam[fp[h]] - lam[fm[h]]);
        }
        if (U != 0.0 || W != 0.0) acc += (wf * U + uf * W) / sf;
        g[f] = -0.5 * acc;
    }
}

__global__ void k_scale_volume(int n, const double* __restrict__ in, const double* __restrict__ vol,
                               double* __restrict__ out, int invert) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = vol[i];
        out[i] = invert ? (v > 0 ? in[i] / v : 0.0) : in[i] * v;
    }
}

int grid_cap(int64_t n) {
    int64_t g = (n + kThreads - 1) / kThreads;
    if (g > 1184) g = 1184;
    return int(g < 1 ? 1 : g);
}

}  // namespace

void DeviceSolver::upload_faces(const Mesh& mesh, const Metric& metric, const std::vector<double>& kappa) {
    TPA_CUDA(cudaSetDevice(device_));
    const int64_t nf = mesh.nfaces();
    if (nf >= (int64_t(1) << 31)) throw Error(5, "too many faces for the adjoint kernels");
    if (int64_t(kappa.size()) != nf) throw Error(1, "one face coefficient is required per interior face");
    // CSR rows of K: the diagonal first, then the off-diagonal entries of the row
    std::vector<int> ptr(size_t(nf) + 1, 0);
    for (size_t e = 0; e < metric.off_row.size(); ++e) ++ptr[size_t(metric.off_row[e]) + 1];
    for (int64_t f = 0; f < nf; ++f) ptr[size_t(f) + 1] += ptr[size_t(f)] + 1;
    std::vector<int> col(static_cast<size_t>(ptr[static_cast<size_t>(nf)]));
    std::vector<double> val(col.size());
    std::vector<int> fill(ptr.begin(), ptr.end() - 1);
    for (int64_t f = 0; f < nf; ++f) {
        col[size_t(fill[size_t(f)])] = int(f);
        val[size_t(fill[size_t(f)]++)] = metric.diag[size_t(f)];
    }
    for (size_t e = 0; e < metric.off_row.size(); ++e) {
        const int r = metric.off_row[e];
        col[size_t(fill[size_t(r)])] = metric.off_col[e];
        val[size_t(fill[size_t(r)]++)] = metric.off_val[e];
    }
    std::vector<double> sk(static_cast<size_t>(nf));
    for (int64_t f = 0; f < nf; ++f) {
        if (!(kappa[size_t(f)] >= 0) || !std::isfinite(kappa[size_t(f)]))
            throw Error(1, "face coefficients must be finite and nonnegative");
        sk[size_t(f)] = std::sqrt(kappa[size_t(f)]);
    }
    // a row with off-diagonal couplings needs kappa_f > 0 for the gradient (the
    // derivative of sqrt(kappa_f) is unbounded at 0)
    hang_zero_ = false;
    for (int64_t f = 0; f < nf; ++f)
        if (ptr[size_t(f) + 1] - ptr[size_t(f)] > 1 && sk[size_t(f)] == 0) hang_zero_ = true;
    std::vector<int> fm(mesh.fm.begin(), mesh.fm.end()), fp(mesh.fp.begin(), mesh.fp.end());
    f_minus_.upload(fm.data(), fm.size(), stream_);
    f_plus_.upload(fp.data(), fp.size(), stream_);
    f_area_.upload(mesh.farea.data(), mesh.farea.size(), stream_);
    k_ptr_.upload(ptr.data(), ptr.size(), stream_);
    k_col_.upload(col.data(), col.size(), stream_);
    k_val_.upload(val.data(), val.size(), stream_);
    f_sqrtk_.upload(sk.data(), sk.size(), stream_);
    TPA_CUDA(cudaStreamSynchronize(stream_));
    nfaces_ = nf;
    nbfaces_ = -1;  // the projection topology follows the faces
}

void DeviceSolver::face_gradient(const double* p, const double* lam, double* g) {
    if (nfaces_ < 0) throw Error(7, "face data not uploaded");
    if (hang_zero_)
        throw Error(1, "the face-coefficient gradient needs kappa > 0 on faces of hanging-vertex patches");
    TPA_CUDA(cudaSetDevice(device_));
    if (nfaces_ == 0) return;
    k_face_gradient<<<grid_cap(nfaces_), kThreads, 0, stream_>>>(int(nfaces_), f_minus_.p, f_plus_.p, f_area_.p,
                                                                 k_ptr_.p, k_col_.p, k_val_.p, f_sqrtk_.p, p, lam,
                                                                 g);
    TPA_CUDA(cudaGetLastError());
    ++launches_;
}

void DeviceSolver::scale_by_volume(const double* in, double* out, bool invert) {
    TPA_CUDA(cudaSetDevice(device_));
    const int n = ncells();
    k_scale_volume<<<grid_cap(n), kThreads, 0, stream_>>>(n, in, levels_[0].d.vol.p, out, invert ? 1 : 0);
    TPA_CUDA(cudaGetLastError());
    ++launches_;
}

}  // namespace tpa
