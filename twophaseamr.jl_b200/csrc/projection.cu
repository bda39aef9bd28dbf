// The one-velocity projection step around the pressure solve, on the device:
// `_project_prepared!` (src/navier_stokes/projection.jl:221-260 of
// ronaldremmerswaal/TwoPhaseAMR.jl) with `divergence!`
// (src/operators/advection/cell_advection.jl:205-220), `_projection_rhs!`
// (projection.jl:130-156), `weighted_gradient!` (src/operators/elliptic.jl:
// 1255-1297), the velocity update and `_accumulate_pressure_increment!`
// (projection.jl:56-98); and the two-phase inputs of a step:
// `_refresh_conditional_fraction!` without embedded geometry
// (src/interface/interface_field.jl:248-291), the face coefficient 1/rho_f
// (src/two_phase/forces.jl:23-36, 69-84, 113-140) and the CSF / CGFM surface
// tension with a constant curvature (forces.jl:179-209, 312-314, 345-378).
//
// Elementwise arithmetic keeps the reference's order of operations with no
// fused multiply-add (explicit round-to-nearest intrinsics), and the
// divergence sums each cell's contributions in face order, so these results
// equal a sequential CPU evaluation bit for bit.  The metric product K v runs
// over K's rows (diagonal first).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "device.cuh"

namespace tpa {

namespace {

constexpr int kPThreads = 256;

int pgrid(int64_t n) {
    int64_t g = (n + kPThreads - 1) / kPThreads;
    return int(std::max<int64_t>(1, std::min<int64_t>(g, 1184)));
}

// physical fraction clamped to [0, 1] and the conditional fraction with the
// floor; err = 1 when a raw value is not finite or beyond 128 eps of [0, 1]
__global__ void kp_conditional(int n, const double* __restrict__ raw, double floor, double* __restrict__ physical,
                               double* __restrict__ conditional, int* err) {
    const double tol = 128.0 * 2.220446049250313e-16;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double r = raw[i];
        if (!(isfinite(r) && r >= -tol && r <= 1.0 + tol)) atomicExch(err, 1);
        double v = fmin(fmax(r, 0.0), 1.0);
        double q = v;  // open fraction 1
        if (q <= floor) {
            v = 0.0;
            q = 0.0;
        } else if (q >= 1.0 - floor) {
            v = 1.0;
            q = 1.0;
        }
        if (physical) physical[i] = v;
        conditional[i] = q;
    }
}

// kappa_f = 1 / (rho_l c + rho_g (1 - c)), c = clamp((hm cm + hp cp) / (hm + hp), 0, 1)
__global__ void kp_face_coefficient(int nf, const int* __restrict__ fm, const int* __restrict__ fp,
                                    const double* __restrict__ hm, const double* __restrict__ hp,
                                    const double* __restrict__ cond, double rho_l, double rho_g,
                                    double* __restrict__ kappa) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
        const double a = hm[f], b = hp[f];
        const double num = __dadd_rn(__dmul_rn(a, cond[fm[f]]), __dmul_rn(b, cond[fp[f]]));
        const double c = fmin(fmax(__ddiv_rn(num, __dadd_rn(a, b)), 0.0), 1.0);
        const double rho = __dadd_rn(__dmul_rn(rho_l, c), __dmul_rn(rho_g, __dsub_rn(1.0, c)));
        kappa[f] = __ddiv_rn(1.0, rho);
    }
}

// in_f = sqrt(k_f) j_f with either the surface-tension jump (mode 0 CGFM,
// 1 CSF; sigma kappa jump |f|, zero when sigma or the jump is zero) or the
// pressure jump |f| (p+ - p-) (mode 2)
__global__ void kp_face_in(int nf, int mode, const int* __restrict__ fm, const int* __restrict__ fp,
                           const double* __restrict__ area, const double* __restrict__ sk,
                           const double* __restrict__ v, double sigma, double curvature, double* __restrict__ in) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
        const double vm = v[fm[f]], vp = v[fp[f]];
        double j;
        if (mode == 2) {
            j = __dmul_rn(area[f], __dsub_rn(vp, vm));
        } else {
            const double jump = mode == 0 ? double(int(vp > 0.5) - int(vm > 0.5)) : __dsub_rn(vp, vm);
            j = (sigma == 0.0 || jump == 0.0) ? 0.0 : __dmul_rn(__dmul_rn(__dmul_rn(sigma, curvature), jump), area[f]);
        }
        in[f] = __dmul_rn(sk[f], j);
    }
}

// out_f = sqrt(k_f) (K in)_f; g[f] = out_f and / or u[f] -= dt out_f
__global__ void kp_face_out(int nf, const int* __restrict__ kptr, const int* __restrict__ kcol,
                            const double* __restrict__ kval, const double* __restrict__ in,
                            const double* __restrict__ sk, double* __restrict__ g, double* __restrict__ u, double dt) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
        int k = kptr[f];
        double s = __dmul_rn(kval[k], in[kcol[k]]);
        for (++k; k < kptr[f + 1]; ++k) s = __dadd_rn(s, __dmul_rn(kval[k], in[kcol[k]]));
        const double w = __dmul_rn(sk[f], s);
        if (g) g[f] = w;
        if (u) u[f] = __dsub_rn(u[f], __dmul_rn(dt, w));
    }
}

// boundary faces of the weighted gradient, `_elliptic_boundary_gradient!`
// (elliptic.jl:1254-1262): -side * (2 k_b / h) * p on open faces, -side * 0 * p
// on closed ones, and the velocity update u_b -= dt g_b; zero = 1 writes the
// zero force instead
__global__ void kp_boundary(int nb, const int* __restrict__ bcell, const double* __restrict__ bside,
                            const double* __restrict__ bgrad, const double* __restrict__ p, double* __restrict__ g,
                            double* __restrict__ u, double dt, int zero) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x) {
        const double w = zero ? 0.0 : __dmul_rn(__dmul_rn(-bside[k], bgrad[k]), p[bcell[k]]);
        if (g) g[k] = w;
        if (u) u[k] = __dsub_rn(u[k], __dmul_rn(dt, w));
    }
}

// per cell, in face order: + u|f|/V (minus side), (-u|f|)/V (plus side),
// (side u_b |f|)/V (boundary); then out = div, or the projection right-hand
// side -div / dt (+ weight * inherited)
__global__ void kp_divergence(int n, int nf, const int* __restrict__ iptr, const int* __restrict__ icode,
                              const double* __restrict__ u, const double* __restrict__ ub,
                              const double* __restrict__ area, const double* __restrict__ barea,
                              const double* __restrict__ bside, const double* __restrict__ vol, int rhs, double dt,
                              const double* __restrict__ inherited, double weight, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double V = vol[i];
        double s = 0.0;
        for (int e = iptr[i]; e < iptr[i + 1]; ++e) {
            const int c = icode[e];
            double t;
            if (c < 2 * nf) {
                const int f = c >> 1;
                const double flux = __dmul_rn(u[f], area[f]);
                t = __ddiv_rn((c & 1) ? -flux : flux, V);
            } else {
                const int k = c - 2 * nf;
                t = __ddiv_rn(__dmul_rn(__dmul_rn(bside[k], ub[k]), barea[k]), V);
            }
            s = __dadd_rn(s, t);
        }
        if (rhs) {
            s = __ddiv_rn(-s, dt);
            if (inherited) s = __dadd_rn(s, __dmul_rn(weight, inherited[i]));
        }
        out[i] = s;
    }
}

__global__ void kp_add(int n, double* __restrict__ p, const double* __restrict__ phi) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = __dadd_rn(p[i], phi[i]);
}

// per-component volume sums of p on split domains (fixed order: per thread,
// then a fixed tree per block); partial[s * gridDim.x + block]
__global__ void kp_slot_partial(int n, const double* __restrict__ p, const double* __restrict__ vol,
                                const int* __restrict__ slot, int ncomp, double* __restrict__ partial) {
    __shared__ double sh[kMaxComponents][kPThreads / 32];
    double acc[kMaxComponents];
    for (int s = 0; s < ncomp; ++s) acc[s] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int s = slot[i];
        if (s >= 0 && s < ncomp) acc[s] += vol[i] * p[i];
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int s = 0; s < ncomp; ++s) {
        double v = acc[s];
        for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (!lane) sh[s][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < ncomp) {
        double v = 0.0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) v += sh[threadIdx.x][w];
        partial[threadIdx.x * gridDim.x + blockIdx.x] = v;
    }
}

// p -= sum_s / volume_s on every cell of component s; cells of no component: 0
__global__ void kp_slot_apply(int n, double* __restrict__ p, const int* __restrict__ slot, int ncomp,
                              const double* __restrict__ partial, int nblocks, const double* __restrict__ cvol) {
    __shared__ double mean[kMaxComponents];
    if (threadIdx.x < ncomp) {
        double v = 0.0;
        for (int b = 0; b < nblocks; ++b) v += partial[threadIdx.x * nblocks + b];
        mean[threadIdx.x] = v / cvol[threadIdx.x];
    }
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int s = slot[i];
        p[i] = (s >= 0 && s < ncomp) ? p[i] - mean[s] : 0.0;
    }
}

}  // namespace

// `enforce_no_permeation!` of the closed sides only: the normal velocity of
// every boundary face that is not on an open side is zeroed (open faces keep
// theirs, `preserve_open`)
__global__ void kp_close_walls(int nb, const unsigned char* __restrict__ open, double* __restrict__ u) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nb; k += gridDim.x * blockDim.x)
        if (!open[k]) u[k] = 0.0;
}

void DeviceSolver::upload_projection(const Mesh& mesh, const std::vector<double>& bgrad,
                                     const std::vector<unsigned char>& open) {
    TPA_CUDA(cudaSetDevice(device_));
    if (nfaces_ < 0) throw Error(7, "face data not uploaded");
    const int64_t nf = mesh.nfaces(), nb = int64_t(mesh.bcell.size()), n = mesh.ncells();
    if (2 * (nf + nb) >= (int64_t(1) << 31)) throw Error(5, "too many faces for the projection kernels");
    // per cell its incident faces in face order: interior (2 f + plus), then
    // boundary (2 nf + k)
    std::vector<int> ptr(size_t(n) + 1, 0);
    for (int64_t f = 0; f < nf; ++f) {
        ++ptr[size_t(mesh.fm[size_t(f)]) + 1];
        ++ptr[size_t(mesh.fp[size_t(f)]) + 1];
    }
    for (int64_t k = 0; k < nb; ++k) ++ptr[size_t(mesh.bcell[size_t(k)]) + 1];
    for (int64_t c = 0; c < n; ++c) ptr[size_t(c) + 1] += ptr[size_t(c)];
    std::vector<int> code(static_cast<size_t>(ptr[size_t(n)])), nxt(ptr.begin(), ptr.end() - 1);
    for (int64_t f = 0; f < nf; ++f) {
        code[size_t(nxt[size_t(mesh.fm[size_t(f)])]++)] = int(2 * f);
        code[size_t(nxt[size_t(mesh.fp[size_t(f)])]++)] = int(2 * f + 1);
    }
    for (int64_t k = 0; k < nb; ++k) code[size_t(nxt[size_t(mesh.bcell[size_t(k)])]++)] = int(2 * nf + k);
    // spacing of the two cells along the face normal
    const int64_t cpb = mesh.cells_per_block();
    std::vector<double> hm(static_cast<size_t>(nf)), hp(static_cast<size_t>(nf)), side(static_cast<size_t>(nb));
    for (int64_t f = 0; f < nf; ++f) {
        const auto& h = mesh.fax[size_t(f)] == 1 ? mesh.bsx : mesh.bsy;
        hm[size_t(f)] = h[size_t(mesh.fm[size_t(f)] / cpb)];
        hp[size_t(f)] = h[size_t(mesh.fp[size_t(f)] / cpb)];
    }
    std::vector<int> bcell(mesh.bcell.begin(), mesh.bcell.end());
    for (int64_t k = 0; k < nb; ++k) side[size_t(k)] = double(mesh.bside[size_t(k)]);
    inc_ptr_.upload(ptr.data(), ptr.size(), stream_);
    inc_code_.upload(code.data(), code.size(), stream_);
    f_hm_.upload(hm.data(), hm.size(), stream_);
    f_hp_.upload(hp.data(), hp.size(), stream_);
    b_cell_.upload(bcell.data(), bcell.size(), stream_);
    b_side_.upload(side.data(), side.size(), stream_);
    b_area_.upload(mesh.barea.data(), mesh.barea.size(), stream_);
    if (bgrad.size() != size_t(nb) || open.size() != size_t(nb)) throw Error(1, "boundary data size mismatch");
    b_grad_.upload(bgrad.data(), bgrad.size(), stream_);
    b_open_.upload(open.data(), open.size(), stream_);
    proj_b_.alloc(size_t(n));
    proj_phi_.alloc(size_t(n));
    proj_in_.alloc(size_t(std::max<int64_t>(nf, 1)));
    perr_.alloc(1);
    const DevLevel& L = levels_[0];
    if (L.ncomp > 1) {
        proj_part_.alloc(size_t(kMaxComponents) * size_t(kReduceBlocks));
        proj_cvol_.upload(L.comp_volume.data(), L.comp_volume.size(), stream_);
    }
    TPA_CUDA(cudaStreamSynchronize(stream_));
    nbfaces_ = nb;
}

void DeviceSolver::conditional_fraction(const double* raw, double floor, double* physical, double* conditional) {
    TPA_CUDA(cudaSetDevice(device_));
    if (!(std::isfinite(floor) && floor > 0 && floor < 0.5))
        throw Error(1, "fraction_floor must be finite and in (0, 0.5)");
    const int n = ncells();
    int err = 0;
    TPA_CUDA(cudaMemsetAsync(perr_.p, 0, sizeof(int), stream_));
    kp_conditional<<<pgrid(n), kPThreads, 0, stream_>>>(n, raw, floor, physical, conditional, perr_.p);
    TPA_CUDA(cudaGetLastError());
    ++launches_;
    TPA_CUDA(cudaMemcpyAsync(&err, perr_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    TPA_CUDA(cudaStreamSynchronize(stream_));
    if (err) throw Error(1, "volume fractions must be finite and lie in [0, 1]");
}

void DeviceSolver::face_coefficients(const double* conditional, double rho_l, double rho_g, double* kappa) {
    TPA_CUDA(cudaSetDevice(device_));
    if (!(std::isfinite(rho_l) && rho_l > 0 && std::isfinite(rho_g) && rho_g > 0))
        throw Error(1, "phase densities must be finite and positive");
    if (nfaces_ <= 0) return;
    kp_face_coefficient<<<pgrid(nfaces_), kPThreads, 0, stream_>>>(int(nfaces_), f_minus_.p, f_plus_.p, f_hm_.p,
                                                                   f_hp_.p, conditional, rho_l, rho_g, kappa);
    TPA_CUDA(cudaGetLastError());
    ++launches_;
}

void DeviceSolver::surface_tension(const double* conditional, double sigma, double curvature, int csf,
                                   double* a_int, double* a_bnd) {
    TPA_CUDA(cudaSetDevice(device_));
    if (!(std::isfinite(sigma) && sigma >= 0)) throw Error(1, "sigma must be finite and nonnegative");
    if (!std::isfinite(curvature)) throw Error(1, "constant curvature must be finite");
    if (nfaces_ > 0) {
        kp_face_in<<<pgrid(nfaces_), kPThreads, 0, stream_>>>(int(nfaces_), csf ? 1 : 0, f_minus_.p, f_plus_.p,
                                                              f_area_.p, f_sqrtk_.p, conditional, sigma, curvature,
                                                              proj_in_.p);
        kp_face_out<<<pgrid(nfaces_), kPThreads, 0, stream_>>>(int(nfaces_), k_ptr_.p, k_col_.p, k_val_.p,
                                                               proj_in_.p, f_sqrtk_.p, a_int, nullptr, 0.0);
        launches_ += 2;
    }
    if (nbfaces_ > 0 && a_bnd) {
        kp_boundary<<<pgrid(nbfaces_), kPThreads, 0, stream_>>>(int(nbfaces_), b_cell_.p, b_side_.p, b_grad_.p, nullptr,
                                                                a_bnd,
                                                                nullptr, 0.0, 1);
        ++launches_;
    }
    TPA_CUDA(cudaGetLastError());
}

void DeviceSolver::weighted_gradient(const double* p, double* g_int, double* g_bnd, double* u_int, double* u_bnd,
                                     double dt) {
    TPA_CUDA(cudaSetDevice(device_));
    if (nfaces_ > 0) {
        kp_face_in<<<pgrid(nfaces_), kPThreads, 0, stream_>>>(int(nfaces_), 2, f_minus_.p, f_plus_.p, f_area_.p,
                                                              f_sqrtk_.p, p, 0.0, 0.0, proj_in_.p);
        kp_face_out<<<pgrid(nfaces_), kPThreads, 0, stream_>>>(int(nfaces_), k_ptr_.p, k_col_.p, k_val_.p,
                                                               proj_in_.p, f_sqrtk_.p, g_int, u_int, dt);
        launches_ += 2;
    }
    if (nbfaces_ > 0 && (g_bnd || u_bnd)) {
        kp_boundary<<<pgrid(nbfaces_), kPThreads, 0, stream_>>>(int(nbfaces_), b_cell_.p, b_side_.p, b_grad_.p, p,
                                                                g_bnd, u_bnd,
                                                                dt, 0);
        ++launches_;
    }
    TPA_CUDA(cudaGetLastError());
}

void DeviceSolver::divergence(const double* u_int, const double* u_bnd, double* out, bool rhs, double dt,
                              const double* inherited, double weight) {
    TPA_CUDA(cudaSetDevice(device_));
    const int n = ncells();
    kp_divergence<<<pgrid(n), kPThreads, 0, stream_>>>(n, int(nfaces_), inc_ptr_.p, inc_code_.p, u_int, u_bnd,
                                                        f_area_.p, b_area_.p, b_side_.p, levels_[0].d.vol.p,
                                                        rhs ? 1 : 0, dt, inherited, weight, out);
    TPA_CUDA(cudaGetLastError());
    ++launches_;
}

void DeviceSolver::project(double* u_int, double* u_bnd, double* p, double dt, double tolerance, int max_cycles,
                           int compatibility, const double* inherited, double reference_dt, int precision,
                           bool prepared, SolveStats& st) {
    TPA_CUDA(cudaSetDevice(device_));
    if (!(dt > 0) || !std::isfinite(dt)) throw Error(1, "dt must be strictly positive");
    if (!(std::isfinite(reference_dt) && reference_dt >= dt))
        throw Error(1, "reference dt must be finite and at least dt");
    if (!(std::isfinite(tolerance) && tolerance > 0 && tolerance < 1))
        throw Error(1, "tolerance must be finite and lie in (0, 1)");
    const int n = ncells();
    // `project!` without a velocity boundary: no permeation through the walls
    if (!prepared && nbfaces_ > 0) {
        if (open_sides_) {
            kp_close_walls<<<pgrid(nbfaces_), kPThreads, 0, stream_>>>(int(nbfaces_), b_open_.p, u_bnd);
            ++launches_;
        } else {
            TPA_CUDA(cudaMemsetAsync(u_bnd, 0, sizeof(double) * size_t(nbfaces_), stream_));
        }
    }
    const double weight = (reference_dt - dt) / (dt * reference_dt);
    divergence(u_int, u_bnd, proj_b_.p, true, dt, inherited, weight);
    TPA_CUDA(cudaMemsetAsync(proj_phi_.p, 0, sizeof(double) * size_t(n), stream_));
    solve(proj_b_.p, proj_phi_.p, 0.0, tolerance / (dt * dt), max_cycles, compatibility, precision, st);
    weighted_gradient(proj_phi_.p, nullptr, nullptr, u_int, u_bnd, dt);  // u -= dt * diffusion * G_k phi
    kp_add<<<pgrid(n), kPThreads, 0, stream_>>>(n, p, proj_phi_.p);
    ++launches_;
    const DevLevel& L = levels_[0];
    if (L.ncomp > 1) {
        kp_slot_partial<<<kReduceBlocks, kPThreads, 0, stream_>>>(n, p, L.d.vol.p, L.slot.p, L.ncomp, proj_part_.p);
        kp_slot_apply<<<pgrid(n), kPThreads, 0, stream_>>>(n, p, L.slot.p, L.ncomp, proj_part_.p, kReduceBlocks,
                                                           proj_cvol_.p);
        launches_ += 2;
    }
    TPA_CUDA(cudaGetLastError());
}

}  // namespace tpa
