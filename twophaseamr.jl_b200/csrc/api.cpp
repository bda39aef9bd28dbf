// C-ABI of the B200 pressure solver (declared in include/tpagmg.h).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/tpagmg.h"
#include "batch.hpp"
#include "cmdgfm.cuh"
#include "device.cuh"
#include "host.hpp"

struct tpa_context {
    int device = 0;
    std::string error;
    bool have_mesh = false, have_operator = false, have_hierarchy = false, uploaded = false;
    tpa::Mesh mesh;
    tpa::LevelOperator op;  // fine operator before the hierarchy takes it
    tpa::Hierarchy hier;
    std::unique_ptr<tpa::DeviceSolver> dev;
    tpa::DevArray<double> d_rhs, d_x, d_y, d_aux, d_face;
    void* user_stream = nullptr;
    // after a device refresh the host copy of the hierarchy beyond the finest
    // face coefficients is out of date; host readers recompute it first
    bool host_stale = false;
    int refresh_path = 0;  // 1 host, 2 device (tpa_last_refresh)
    double refresh_ms = 0;
    // open sides (left, right, bottom, top) and their explicit boundary
    // coefficients (empty: extended from the interior ones)
    bool open[4] = {false, false, false, false};
    std::vector<double> bcoef;
    std::unique_ptr<tpa::CmdgfmDevice> cmdgfm;  // vectors of the CMDGFM solve, kept between calls
};

namespace tpa {
void set_context_error(tpa_context* ctx, const std::string& msg) { ctx->error = msg; }
}  // namespace tpa

namespace {

template <typename F>
tpa_status guard(tpa_context* ctx, F&& f) {
    if (!ctx) return TPA_ERR_INVALID_ARG;
    try {
        ctx->error.clear();
        f();
        return TPA_OK;
    } catch (const tpa::Error& e) {
        ctx->error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        ctx->error = "host allocation failed";
        return TPA_ERR_INVALID_ARG;
    } catch (const std::exception& e) {
        ctx->error = e.what();
        return TPA_ERR_INVALID_ARG;
    }
}

// the context's open sides on a fine operator (kappa set): explicit boundary
// coefficients, or the interior ones extended (`_boundary_material`)
void apply_open_sides(const tpa_context* ctx, tpa::LevelOperator& op) {
    std::copy(ctx->open, ctx->open + 4, op.open);
    if (!op.any_open()) {
        op.bkappa.assign(op.mesh.bcell.size(), 0.0);
        return;
    }
    if (!ctx->bcoef.empty()) op.bkappa = ctx->bcoef;
    else tpa::extend_boundary_material(op);
}

const tpa::LevelOperator& fine_op(const tpa_context* ctx) {
    if (ctx->have_hierarchy) return ctx->hier.levels[0].op;
    if (!ctx->have_operator) throw tpa::Error(TPA_ERR_STATE, "no operator: call tpa_set_operator first");
    return ctx->op;
}

void ensure_host_fresh(tpa_context* ctx) {
    if (!ctx->host_stale) return;
    tpa::refresh_hierarchy(ctx->hier, ctx->hier.levels[0].op.kappa);
    ctx->host_stale = false;
}

void ensure_device(tpa_context* ctx) {
    if (!ctx->have_hierarchy) throw tpa::Error(TPA_ERR_STATE, "no hierarchy: call tpa_build_hierarchy first");
    if (ctx->uploaded) return;
    ensure_host_fresh(ctx);
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count <= ctx->device)
        throw tpa::Error(TPA_ERR_CUDA, "no usable CUDA device for the B200 solver");
    if (!ctx->dev) ctx->dev.reset(new tpa::DeviceSolver(ctx->device));
    ctx->dev->set_stream(static_cast<cudaStream_t>(ctx->user_stream));
    ctx->dev->upload(ctx->hier);
    ctx->dev->invalidate_faces();
    size_t n = size_t(ctx->dev->ncells());
    ctx->d_rhs.alloc(n);
    ctx->d_x.alloc(n);
    ctx->d_y.alloc(n);
    ctx->uploaded = true;
}

void ensure_faces(tpa_context* ctx) {
    ensure_device(ctx);
    if (!ctx->dev->faces_ready()) {
        const tpa::LevelOperator& op = ctx->hier.levels[0].op;
        ctx->dev->upload_faces(op.mesh, op.metric, op.kappa);
    }
}

void ensure_projection(tpa_context* ctx) {
    ensure_faces(ctx);
    if (!ctx->dev->projection_ready()) {
        const tpa::LevelOperator& op = ctx->hier.levels[0].op;
        std::vector<unsigned char> open(op.mesh.bcell.size());
        for (size_t b = 0; b < open.size(); ++b) open[b] = op.open_face(int64_t(b)) ? 1 : 0;
        ctx->dev->upload_projection(op.mesh, op.bgrad, open);
    }
}

void fill_stats(const tpa::SolveStats& s, int precision, int launches, tpa_stats* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    out->cycles = s.cycles;
    out->converged = s.converged;
    out->compatible = 1;
    out->restarts = s.restarts;
    out->initial_l2 = s.initial_l2;
    out->initial_linf = s.initial_linf;
    out->final_l2 = s.final_l2;
    out->final_linf = s.final_linf;
    out->target_linf = s.target_linf;
    out->residual_scale = s.residual_scale;
    out->removed_rhs_mean = s.removed_rhs_mean;
    out->device_ms = s.ms_total;
    out->kernel_launches = launches;
    out->precision = precision;
    out->removed_rhs_max_component_mean = s.removed_max_component_mean;
}

void solve_host_body(tpa_context* ctx, const double* rhs, double* x, double rtol, double atol, int32_t max_cycles,
                     int32_t compatibility, int32_t precision, tpa_stats* stats) {
    if (!rhs || !x) throw tpa::Error(TPA_ERR_INVALID_ARG, "null rhs or solution");
    ensure_device(ctx);
    size_t n = size_t(ctx->dev->ncells());
    // the fused solve checks the right-hand side on the device (sum |V f| is finite)
    if (!ctx->dev->fused())
        for (size_t i = 0; i < n; ++i)
            if (!std::isfinite(rhs[i])) throw tpa::Error(TPA_ERR_NONFINITE, "right-hand side must be finite");
    cudaStream_t s = ctx->dev->stream();
    TPA_CUDA(cudaMemcpyAsync(ctx->d_rhs.p, rhs, n * sizeof(double), cudaMemcpyHostToDevice, s));
    TPA_CUDA(cudaMemcpyAsync(ctx->d_x.p, x, n * sizeof(double), cudaMemcpyHostToDevice, s));
    tpa::SolveStats st;
    ctx->dev->reset_launches();
    ctx->dev->solve(ctx->d_rhs.p, ctx->d_x.p, rtol, atol, max_cycles, compatibility, precision, st);
    TPA_CUDA(cudaMemcpyAsync(x, ctx->d_x.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    TPA_CUDA(cudaStreamSynchronize(s));
    fill_stats(st, precision, ctx->dev->kernel_launches(), stats);
}

void solve_device_body(tpa_context* ctx, const double* rhs, double* x, double rtol, double atol, int32_t max_cycles,
                       int32_t compatibility, int32_t precision, tpa_stats* stats) {
    if (!rhs || !x) throw tpa::Error(TPA_ERR_INVALID_ARG, "null rhs or solution");
    ensure_device(ctx);
    tpa::SolveStats st;
    ctx->dev->reset_launches();
    ctx->dev->solve(rhs, x, rtol, atol, max_cycles, compatibility, precision, st);
    fill_stats(st, precision, ctx->dev->kernel_launches(), stats);
}

// Independent problems on a pool of host threads, one context (and stream) per
// problem.  device_ms: the device-time span from a start event that every
// problem's stream waits on to the last problem's completion event.
template <typename F>
tpa_status run_batched(tpa_context* const* ctxs, int32_t count, int32_t workers, tpa_status* statuses,
                       double* device_ms, F solve_one) {
    if (count < 0 || (count > 0 && !ctxs)) return TPA_ERR_INVALID_ARG;
    for (int32_t k = 0; k < count; ++k)
        if (!ctxs[k] || ctxs[k]->device != ctxs[0]->device) return TPA_ERR_INVALID_ARG;
    {
        std::vector<tpa_context*> sorted(ctxs, ctxs + count);
        std::sort(sorted.begin(), sorted.end());
        if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end()) return TPA_ERR_INVALID_ARG;
    }
    if (device_ms) *device_ms = 0;
    if (count == 0) return TPA_OK;
    if (workers <= 0) workers = 32;
    workers = std::min(workers, count);
    const int dev = ctxs[0]->device;
    cudaEvent_t start = nullptr;
    std::vector<cudaEvent_t> done(size_t(count), nullptr);
    if (device_ms) {
        if (cudaSetDevice(dev) != cudaSuccess || cudaEventCreate(&start) != cudaSuccess ||
            cudaEventRecord(start, nullptr) != cudaSuccess)
            return TPA_ERR_CUDA;
    }
    std::vector<tpa_status> st(size_t(count), TPA_OK);
    std::atomic<int32_t> next{0};
    auto run = [&] {
        cudaSetDevice(dev);
        for (int32_t k = next++; k < count; k = next++) {
            tpa_context* ctx = ctxs[k];
            st[size_t(k)] = guard(ctx, [&] {
                ensure_device(ctx);
                cudaStream_t s = ctx->dev->stream();
                if (start) TPA_CUDA(cudaStreamWaitEvent(s, start, 0));
                solve_one(ctx, k);
                if (start) {
                    TPA_CUDA(cudaEventCreate(&done[size_t(k)]));
                    TPA_CUDA(cudaEventRecord(done[size_t(k)], s));
                }
            });
        }
    };
    std::vector<std::thread> pool;
    try {
        for (int32_t w = 1; w < workers; ++w) pool.emplace_back(run);
    } catch (...) {
        // fewer threads than asked: the workers that started (and this thread) take every problem
    }
    run();
    for (auto& t : pool) t.join();
    tpa_status first = TPA_OK;
    for (int32_t k = 0; k < count; ++k) {
        if (statuses) statuses[k] = st[size_t(k)];
        if (first == TPA_OK) first = st[size_t(k)];
    }
    if (start) {
        float span = 0;
        for (int32_t k = 0; k < count; ++k) {
            cudaEvent_t e = done[size_t(k)];
            if (!e) continue;
            float ms = 0;
            if (cudaEventSynchronize(e) == cudaSuccess && cudaEventElapsedTime(&ms, start, e) == cudaSuccess)
                span = std::max(span, ms);
            cudaEventDestroy(e);
        }
        cudaEventDestroy(start);
        *device_ms = span;
    }
    return first;
}

}  // namespace

extern "C" {

tpa_status tpa_create(tpa_context** out, int32_t device) {
    if (!out || device < 0) return TPA_ERR_INVALID_ARG;
    try {
        *out = new tpa_context();
        (*out)->device = device;
        return TPA_OK;
    } catch (...) {
        return TPA_ERR_INVALID_ARG;
    }
}

void tpa_destroy(tpa_context* ctx) {
    if (!ctx) return;
    try {
        ctx->d_rhs.free();
        ctx->d_x.free();
        ctx->d_y.free();
        ctx->d_aux.free();
        ctx->d_face.free();
        ctx->dev.reset();
    } catch (...) {
    }
    delete ctx;
}

const char* tpa_last_error(const tpa_context* ctx) { return ctx ? ctx->error.c_str() : "null context"; }

tpa_status tpa_set_mesh(tpa_context* ctx, const int32_t base_mesh[2], const int32_t block_size[2],
                        const int32_t periodic[2], const double origin[2], const double extent[2], int64_t nleaves,
                        const int32_t* leaf_keys) {
    return guard(ctx, [&] {
        if (!base_mesh || !block_size || !periodic || !origin || !extent || (nleaves > 0 && !leaf_keys) ||
            nleaves < 0)
            throw tpa::Error(TPA_ERR_INVALID_ARG, "null argument");
        int base[2] = {base_mesh[0], base_mesh[1]}, bs[2] = {block_size[0], block_size[1]};
        bool per[2] = {periodic[0] != 0, periodic[1] != 0};
        for (int a = 0; a < 2; ++a)
            if (!std::isfinite(origin[a]) || !std::isfinite(extent[a]))
                throw tpa::Error(TPA_ERR_NONFINITE, "domain origin and extent must be finite");
        std::vector<uint64_t> leaves;
        if (nleaves == 0) {
            for (int j = 0; j < base[1] / std::max(bs[1], 1); ++j)
                for (int i = 0; i < base[0] / std::max(bs[0], 1); ++i) leaves.push_back(tpa::pack_key(0, i, j));
        } else {
            for (int64_t k = 0; k < nleaves; ++k) {
                const int32_t* kk = leaf_keys + 3 * k;
                if (kk[0] < 0 || kk[1] < 0 || kk[2] < 0) throw tpa::Error(TPA_ERR_INVALID_ARG, "negative leaf key");
                leaves.push_back(tpa::pack_key(kk[0], kk[1], kk[2]));
            }
        }
        ctx->mesh = tpa::build_mesh(base, bs, per, origin, extent, leaves);
        ctx->have_mesh = true;
        ctx->have_operator = ctx->have_hierarchy = ctx->uploaded = false;
    });
}

tpa_status tpa_mesh_sizes(const tpa_context* cctx, int64_t out[5]) {
    auto* ctx = const_cast<tpa_context*>(cctx);
    return guard(ctx, [&] {
        if (!ctx->have_mesh) throw tpa::Error(TPA_ERR_STATE, "no mesh");
        const tpa::Mesh& m = ctx->have_hierarchy ? ctx->hier.levels[0].op.mesh : ctx->mesh;
        out[0] = m.nblocks();
        out[1] = m.ncells();
        out[2] = m.nfaces();
        out[3] = int64_t(m.bcell.size());
        out[4] = m.active;
    });
}

static const tpa::Mesh& cur_mesh(const tpa_context* ctx) {
    if (!ctx->have_mesh) throw tpa::Error(TPA_ERR_STATE, "no mesh");
    return ctx->have_hierarchy ? ctx->hier.levels[0].op.mesh : (ctx->have_operator ? ctx->op.mesh : ctx->mesh);
}

tpa_status tpa_mesh_blocks(const tpa_context* cctx, int32_t* keys, double* geometry) {
    auto* ctx = const_cast<tpa_context*>(cctx);
    return guard(ctx, [&] {
        const tpa::Mesh& m = cur_mesh(ctx);
        for (int64_t b = 0; b < m.nblocks(); ++b) {
            uint64_t k = m.keys[size_t(b)];
            if (keys) {
                keys[3 * b] = tpa::key_level(k);
                keys[3 * b + 1] = int32_t(tpa::key_i(k));
                keys[3 * b + 2] = int32_t(tpa::key_j(k));
            }
            if (geometry) {
                geometry[5 * b] = m.box[size_t(b)];
                geometry[5 * b + 1] = m.boy[size_t(b)];
                geometry[5 * b + 2] = m.bsx[size_t(b)];
                geometry[5 * b + 3] = m.bsy[size_t(b)];
                geometry[5 * b + 4] = m.bvol[size_t(b)];
            }
        }
    });
}

tpa_status tpa_mesh_faces(const tpa_context* cctx, int32_t* minus, int32_t* plus, int8_t* axis, double* area) {
    auto* ctx = const_cast<tpa_context*>(cctx);
    return guard(ctx, [&] {
        const tpa::Mesh& m = cur_mesh(ctx);
        size_t nf = m.fm.size();
        if (minus) std::memcpy(minus, m.fm.data(), nf * sizeof(int32_t));
        if (plus) std::memcpy(plus, m.fp.data(), nf * sizeof(int32_t));
        if (axis) std::memcpy(axis, m.fax.data(), nf);
        if (area) std::memcpy(area, m.farea.data(), nf * sizeof(double));
    });
}

tpa_status tpa_mesh_boundary_faces(const tpa_context* cctx, int32_t* cell, int8_t* axis, int8_t* side,
                                   double* area) {
    auto* ctx = const_cast<tpa_context*>(cctx);
    return guard(ctx, [&] {
        const tpa::Mesh& m = cur_mesh(ctx);
        size_t nb = m.bcell.size();
        if (cell) std::memcpy(cell, m.bcell.data(), nb * sizeof(int32_t));
        if (axis) std::memcpy(axis, m.bax.data(), nb);
        if (side) std::memcpy(side, m.bside.data(), nb);
        if (area) std::memcpy(area, m.barea.data(), nb * sizeof(double));
    });
}

tpa_status tpa_set_operator(tpa_context* ctx, const double* face_coefficient) {
    return guard(ctx, [&] {
        if (!ctx->have_mesh) throw tpa::Error(TPA_ERR_STATE, "no mesh: call tpa_set_mesh first");
        if (!face_coefficient) throw tpa::Error(TPA_ERR_INVALID_ARG, "null face coefficients");
        tpa::LevelOperator op;
        op.mesh = ctx->have_hierarchy ? ctx->hier.levels[0].op.mesh : (ctx->have_operator ? ctx->op.mesh : ctx->mesh);
        size_t nf = op.mesh.fm.size();
        for (size_t f = 0; f < nf; ++f)
            if (!std::isfinite(face_coefficient[f])) throw tpa::Error(TPA_ERR_NONFINITE, "face coefficients must be finite");
        op.kappa.assign(face_coefficient, face_coefficient + nf);
        op.metric = tpa::assemble_metric(op.mesh);
        apply_open_sides(ctx, op);
        tpa::assemble_operator(op);
        ctx->op = std::move(op);
        ctx->have_operator = true;
        ctx->have_hierarchy = ctx->uploaded = false;
    });
}

tpa_status tpa_set_open_boundaries(tpa_context* ctx, const int32_t open_sides[4], const double* boundary_coefficient) {
    return guard(ctx, [&] {
        if (!ctx->have_mesh) throw tpa::Error(TPA_ERR_STATE, "no mesh: call tpa_set_mesh first");
        if (!open_sides) throw tpa::Error(TPA_ERR_INVALID_ARG, "null open sides");
        const tpa::Mesh& m = ctx->have_hierarchy ? ctx->hier.levels[0].op.mesh
                                                 : (ctx->have_operator ? ctx->op.mesh : ctx->mesh);
        const size_t nb = m.bcell.size();
        std::vector<double> bc;
        if (boundary_coefficient) {
            bc.assign(boundary_coefficient, boundary_coefficient + nb);
            for (double v : bc)
                if (!std::isfinite(v) || v < 0)
                    throw tpa::Error(TPA_ERR_INVALID_ARG, "boundary coefficients must be finite and nonnegative");
        }
        for (int a = 0; a < 2; ++a)
            if (m.periodic[a] && (open_sides[2 * a] || open_sides[2 * a + 1]))
                throw tpa::Error(TPA_ERR_INVALID_ARG, "a periodic axis has no open sides");
        bool open[4];
        for (int k = 0; k < 4; ++k) open[k] = open_sides[k] != 0;
        // a fine operator that exists is assembled again (the hierarchy must be
        // rebuilt): `_update_elliptic_boundary_coefficient!` (elliptic.jl:826-845)
        if (ctx->have_operator || ctx->have_hierarchy) {
            tpa::LevelOperator op = ctx->have_hierarchy ? ctx->hier.levels[0].op : ctx->op;
            std::copy(open, open + 4, ctx->open);
            ctx->bcoef = bc;
            apply_open_sides(ctx, op);
            tpa::assemble_operator(op);
            ctx->op = std::move(op);
            ctx->have_operator = true;
            ctx->have_hierarchy = ctx->uploaded = false;
        } else {
            std::copy(open, open + 4, ctx->open);
            ctx->bcoef = std::move(bc);
        }
    });
}

tpa_status tpa_metric_offdiagonal_count(const tpa_context* cctx, int64_t* count) {
    auto* ctx = const_cast<tpa_context*>(cctx);
    return guard(ctx, [&] { *count = int64_t(fine_op(ctx).metric.off_val.size()); });
}

tpa_status tpa_build_hierarchy(tpa_context* ctx, const tpa_multigrid_options* opts) {
    return guard(ctx, [&] {
        if (!ctx->have_operator && !ctx->have_hierarchy)
            throw tpa::Error(TPA_ERR_STATE, "no operator: call tpa_set_operator first");
        tpa::HierarchyOptions o;
        if (opts) {
            o.coarse_size = opts->coarse_size;
            o.pre_sweeps = opts->pre_sweeps;
            o.post_sweeps = opts->post_sweeps;
            o.max_levels = opts->max_levels;
            o.smoother = opts->smoother;
        }
        if (o.smoother != 0 && o.smoother != 1)
            throw tpa::Error(TPA_ERR_INVALID_ARG, "smoother must be 0 (damped Jacobi) or 1 (red-black Gauss-Seidel)");
        if (o.pre_sweeps != o.post_sweeps)
            throw tpa::Error(TPA_ERR_INVALID_ARG,
                             "CG requires equal pre_sweeps and post_sweeps for a geometric multigrid preconditioner");
        if (ctx->have_hierarchy) ensure_host_fresh(ctx);
        tpa::LevelOperator fine = ctx->have_hierarchy ? ctx->hier.levels[0].op : std::move(ctx->op);
        ctx->have_hierarchy = false;
        ctx->hier = tpa::build_hierarchy(std::move(fine), o);
        ctx->op = tpa::LevelOperator();
        ctx->have_hierarchy = true;
        ctx->have_operator = true;
        ctx->uploaded = false;
        if (ctx->dev) ctx->dev->reset_tuning();  // a new hierarchy starts from the default layout
    });
}

tpa_status tpa_hierarchy_sizes(const tpa_context* cctx, int32_t* nlevels, int64_t* sizes, int32_t capacity) {
    auto* ctx = const_cast<tpa_context*>(cctx);
    return guard(ctx, [&] {
        if (!ctx->have_hierarchy) throw tpa::Error(TPA_ERR_STATE, "no hierarchy");
        int32_t nl = int32_t(ctx->hier.levels.size());
        if (nlevels) *nlevels = nl;
        for (int32_t l = 0; sizes && l < nl && l < capacity; ++l) sizes[l] = ctx->hier.levels[size_t(l)].op.A.n;
    });
}

static const tpa::HostLevel& level_of(const tpa_context* ctx, int32_t level) {
    if (!ctx->have_hierarchy) throw tpa::Error(TPA_ERR_STATE, "no hierarchy");
    if (level < 0 || size_t(level) >= ctx->hier.levels.size()) throw tpa::Error(TPA_ERR_INVALID_ARG, "bad level");
    return ctx->hier.levels[size_t(level)];
}

tpa_status tpa_level_owners(const tpa_context* cctx, int32_t level, int32_t* owners) {
    auto* ctx = const_cast<tpa_context*>(cctx);
    return guard(ctx, [&] {
        const tpa::HostLevel& l = level_of(ctx, level);
        if (l.owner.empty()) throw tpa::Error(TPA_ERR_INVALID_ARG, "the coarsest level has no transfer");
        std::memcpy(owners, l.owner.data(), l.owner.size() * sizeof(int32_t));
    });
}

tpa_status tpa_level_info(const tpa_context* cctx, int32_t level, double* sw, double* tw, int32_t* comps) {
    auto* ctx = const_cast<tpa_context*>(cctx);
    return guard(ctx, [&] {
        ensure_host_fresh(ctx);
        const tpa::HostLevel& l = level_of(ctx, level);
        if (sw) *sw = l.weight;
        if (tw) *tw = l.transfer_weight;
        if (comps) *comps = l.op.singular ? int32_t(l.op.comp.volume.size()) : 0;
    });
}

tpa_status tpa_level_red_black(const tpa_context* cctx, int32_t level, uint8_t* colours, double* weight) {
    auto* ctx = const_cast<tpa_context*>(cctx);
    return guard(ctx, [&] {
        ensure_host_fresh(ctx);
        const tpa::HostLevel& l = level_of(ctx, level);
        std::vector<unsigned char> c = tpa::red_black_colours(l.op.mesh);
        if (colours) std::memcpy(colours, c.data(), c.size());
        if (weight) *weight = tpa::red_black_weight(l.op.A, c);
    });
}

tpa_status tpa_level_face_coefficients(const tpa_context* cctx, int32_t level, double* kappa) {
    auto* ctx = const_cast<tpa_context*>(cctx);
    return guard(ctx, [&] {
        ensure_host_fresh(ctx);
        const tpa::HostLevel& l = level_of(ctx, level);
        std::memcpy(kappa, l.op.kappa.data(), l.op.kappa.size() * sizeof(double));
    });
}

tpa_status tpa_level_matrix(const tpa_context* cctx, int32_t level, int64_t* nnz, int64_t* row_ptr, int32_t* col,
                            double* val) {
    auto* ctx = const_cast<tpa_context*>(cctx);
    return guard(ctx, [&] {
        if (!nnz) throw tpa::Error(TPA_ERR_INVALID_ARG, "null output");
        ensure_host_fresh(ctx);
        const tpa::Csr& a = level_of(ctx, level).op.A;
        *nnz = int64_t(a.col.size());
        if (row_ptr) std::memcpy(row_ptr, a.ptr.data(), a.ptr.size() * sizeof(int64_t));
        if (col) std::memcpy(col, a.col.data(), a.col.size() * sizeof(int32_t));
        if (val) std::memcpy(val, a.val.data(), a.val.size() * sizeof(double));
    });
}

tpa_status tpa_last_refresh(const tpa_context* cctx, int32_t* path, double* ms) {
    auto* ctx = const_cast<tpa_context*>(cctx);
    return guard(ctx, [&] {
        if (path) *path = ctx->refresh_path;
        if (ms) *ms = ctx->refresh_ms;
    });
}

tpa_status tpa_refresh(tpa_context* ctx, const double* face_coefficient) {
    const auto t0 = std::chrono::steady_clock::now();
    auto stamp = [&](int path) {
        ctx->refresh_path = path;
        ctx->refresh_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };
    return guard(ctx, [&] {
        if (!ctx->have_hierarchy) throw tpa::Error(TPA_ERR_STATE, "no hierarchy");
        size_t nf = ctx->hier.levels[0].op.kappa.size();
        for (size_t f = 0; f < nf; ++f)
            if (!std::isfinite(face_coefficient[f]) || face_coefficient[f] < 0)
                throw tpa::Error(TPA_ERR_INVALID_ARG, "face coefficients must be finite and nonnegative");
        // the device path keeps the sparsity and the components, so the set of
        // zero coefficients must not change
        const std::vector<double>& old = ctx->hier.levels[0].op.kappa;
        bool same_zeros = old.size() == nf;
        for (size_t f = 0; same_zeros && f < nf; ++f) same_zeros = (face_coefficient[f] == 0) == (old[f] == 0);
        if (ctx->uploaded && same_zeros && !std::getenv("TPAGMG_HOST_REFRESH") &&
            ctx->dev->refresh_applicable(ctx->hier)) {
            try {
                ctx->dev->refresh_on_device(ctx->hier, face_coefficient);
                ctx->hier.levels[0].op.kappa.assign(face_coefficient, face_coefficient + nf);
                ctx->host_stale = true;
                stamp(2);
                return;
            } catch (const tpa::Error&) {
                // the host path below reports the same condition; the device copy
                // is re-uploaded from the host hierarchy
                ctx->uploaded = false;
            }
        }
        tpa::refresh_hierarchy(ctx->hier, std::vector<double>(face_coefficient, face_coefficient + nf));
        ctx->host_stale = false;
        if (ctx->uploaded) {
            ctx->dev->upload(ctx->hier);
            ctx->dev->invalidate_faces();
        }
        stamp(1);
    });
}

tpa_status tpa_refresh_device(tpa_context* ctx, const double* face_coefficient) {
    const auto t0 = std::chrono::steady_clock::now();
    auto stamp = [&](int path) {
        ctx->refresh_path = path;
        ctx->refresh_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    };
    return guard(ctx, [&] {
        if (!face_coefficient) throw tpa::Error(TPA_ERR_INVALID_ARG, "null face coefficients");
        ensure_device(ctx);
        std::vector<double>& kappa = ctx->hier.levels[0].op.kappa;
        const size_t nf = kappa.size();
        cudaStream_t s = ctx->dev->stream();
        if (!std::getenv("TPAGMG_HOST_REFRESH") && ctx->dev->refresh_applicable(ctx->hier) &&
            ctx->dev->refresh_from_device(ctx->hier, face_coefficient) == 0) {
            // the host keeps the finest coefficients (the rest is recomputed on demand)
            TPA_CUDA(cudaMemcpyAsync(kappa.data(), face_coefficient, nf * sizeof(double), cudaMemcpyDeviceToHost, s));
            TPA_CUDA(cudaStreamSynchronize(s));
            ctx->host_stale = true;
            stamp(2);
            return;
        }
        std::vector<double> k(nf);
        TPA_CUDA(cudaMemcpyAsync(k.data(), face_coefficient, nf * sizeof(double), cudaMemcpyDeviceToHost, s));
        TPA_CUDA(cudaStreamSynchronize(s));
        for (size_t f = 0; f < nf; ++f)
            if (!std::isfinite(k[f]) || k[f] < 0)
                throw tpa::Error(TPA_ERR_INVALID_ARG, "face coefficients must be finite and nonnegative");
        tpa::refresh_hierarchy(ctx->hier, k);
        ctx->host_stale = false;
        ctx->dev->upload(ctx->hier);
        ctx->dev->invalidate_faces();
        stamp(1);
    });
}

tpa_status tpa_solve_device(tpa_context* ctx, const double* rhs, double* x, double rtol, double atol,
                            int32_t max_cycles, int32_t compatibility, int32_t precision, tpa_stats* stats) {
    return guard(ctx, [&] { solve_device_body(ctx, rhs, x, rtol, atol, max_cycles, compatibility, precision, stats); });
}

tpa_status tpa_solve(tpa_context* ctx, const double* rhs, double* x, double rtol, double atol, int32_t max_cycles,
                     int32_t compatibility, int32_t precision, tpa_stats* stats) {
    return guard(ctx, [&] { solve_host_body(ctx, rhs, x, rtol, atol, max_cycles, compatibility, precision, stats); });
}

tpa_status tpa_solve_batched(tpa_context* const* ctxs, int32_t count, const double* const* rhs, double* const* x,
                             double rtol, double atol, int32_t max_cycles, int32_t compatibility, int32_t precision,
                             int32_t workers, tpa_stats* stats, tpa_status* statuses, double* device_ms) {
    if (count > 0 && (!rhs || !x)) return TPA_ERR_INVALID_ARG;
    return run_batched(ctxs, count, workers, statuses, device_ms, [&](tpa_context* ctx, int32_t k) {
        solve_host_body(ctx, rhs[k], x[k], rtol, atol, max_cycles, compatibility, precision,
                        stats ? stats + k : nullptr);
    });
}

tpa_status tpa_solve_batched_device(tpa_context* const* ctxs, int32_t count, const double* const* rhs,
                                    double* const* x, double rtol, double atol, int32_t max_cycles,
                                    int32_t compatibility, int32_t precision, int32_t workers, tpa_stats* stats,
                                    tpa_status* statuses, double* device_ms) {
    if (count > 0 && (!rhs || !x)) return TPA_ERR_INVALID_ARG;
    return run_batched(ctxs, count, workers, statuses, device_ms, [&](tpa_context* ctx, int32_t k) {
        solve_device_body(ctx, rhs[k], x[k], rtol, atol, max_cycles, compatibility, precision,
                          stats ? stats + k : nullptr);
    });
}

tpa_status tpa_apply(tpa_context* ctx, const double* x, double* y) {
    return guard(ctx, [&] {
        ensure_device(ctx);
        size_t n = size_t(ctx->dev->ncells());
        cudaStream_t s = ctx->dev->stream();
        TPA_CUDA(cudaMemcpyAsync(ctx->d_x.p, x, n * sizeof(double), cudaMemcpyHostToDevice, s));
        ctx->dev->apply(ctx->d_x.p, ctx->d_y.p);
        TPA_CUDA(cudaMemcpyAsync(y, ctx->d_y.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        TPA_CUDA(cudaStreamSynchronize(s));
    });
}

tpa_status tpa_vcycle(tpa_context* ctx, const double* r, double* z, int32_t precision) {
    return guard(ctx, [&] {
        if (precision != 0 && precision != 1) throw tpa::Error(TPA_ERR_INVALID_ARG, "bad precision");
        ensure_device(ctx);
        size_t n = size_t(ctx->dev->ncells());
        cudaStream_t s = ctx->dev->stream();
        TPA_CUDA(cudaMemcpyAsync(ctx->d_x.p, r, n * sizeof(double), cudaMemcpyHostToDevice, s));
        ctx->dev->vcycle(ctx->d_x.p, ctx->d_y.p, precision);
        TPA_CUDA(cudaMemcpyAsync(z, ctx->d_y.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        TPA_CUDA(cudaStreamSynchronize(s));
        ctx->dev->check_barrier();
    });
}

tpa_status tpa_face_coefficient_gradient(tpa_context* ctx, const double* p, const double* lam, double* grad) {
    return guard(ctx, [&] {
        if (!p || !lam || !grad) throw tpa::Error(TPA_ERR_INVALID_ARG, "null argument");
        ensure_faces(ctx);
        size_t n = size_t(ctx->dev->ncells()), nf = size_t(ctx->dev->nfaces());
        if (ctx->d_face.n != nf) ctx->d_face.alloc(nf);
        cudaStream_t s = ctx->dev->stream();
        TPA_CUDA(cudaMemcpyAsync(ctx->d_x.p, p, n * sizeof(double), cudaMemcpyHostToDevice, s));
        TPA_CUDA(cudaMemcpyAsync(ctx->d_y.p, lam, n * sizeof(double), cudaMemcpyHostToDevice, s));
        ctx->dev->face_gradient(ctx->d_x.p, ctx->d_y.p, ctx->d_face.p);
        TPA_CUDA(cudaMemcpyAsync(grad, ctx->d_face.p, nf * sizeof(double), cudaMemcpyDeviceToHost, s));
        TPA_CUDA(cudaStreamSynchronize(s));
    });
}

static void adjoint_on_device(tpa_context* ctx, const double* p, const double* pbar, double* rhs_bar,
                              double* kappa_bar, double rtol, double atol, int32_t max_cycles, int32_t precision,
                              tpa_stats* stats) {
    // Open sides: the operator stays symmetric and an anchored component has
    // no projection and no gauge, so the adjoint solve is the solve.  The
    // gradient is taken at fixed boundary coefficients, as a coefficient
    // refresh keeps them (`_replace_face_coefficient`, elliptic.jl:809-824):
    // the open-face conductances then do not depend on kappa, and the face
    // kernel's -lam' (dS/dkappa_f) p is the whole derivative.
    ensure_faces(ctx);
    tpa::DeviceSolver& d = *ctx->dev;
    size_t n = size_t(d.ncells());
    if (ctx->d_aux.n != n) ctx->d_aux.alloc(n);
    cudaStream_t s = d.stream();
    d.reset_launches();
    // strong right-hand side pbar / V, zero initial adjoint state
    d.scale_by_volume(pbar, ctx->d_rhs.p, true);
    TPA_CUDA(cudaMemsetAsync(ctx->d_aux.p, 0, n * sizeof(double), s));
    tpa::SolveStats st;
    d.solve(ctx->d_rhs.p, ctx->d_aux.p, rtol, atol, max_cycles, 0, precision, st);
    if (rhs_bar) d.scale_by_volume(ctx->d_aux.p, rhs_bar, false);
    if (kappa_bar) d.face_gradient(p, ctx->d_aux.p, kappa_bar);
    fill_stats(st, precision, d.kernel_launches(), stats);
}

tpa_status tpa_adjoint_device(tpa_context* ctx, const double* p, const double* pbar, double* rhs_bar,
                              double* kappa_bar, double rtol, double atol, int32_t max_cycles, int32_t precision,
                              tpa_stats* stats) {
    return guard(ctx, [&] {
        if (!p || !pbar) throw tpa::Error(TPA_ERR_INVALID_ARG, "null solution or cotangent");
        adjoint_on_device(ctx, p, pbar, rhs_bar, kappa_bar, rtol, atol, max_cycles, precision, stats);
    });
}

tpa_status tpa_adjoint(tpa_context* ctx, const double* p, const double* pbar, double* rhs_bar, double* kappa_bar,
                       double rtol, double atol, int32_t max_cycles, int32_t precision, tpa_stats* stats) {
    return guard(ctx, [&] {
        if (!p || !pbar) throw tpa::Error(TPA_ERR_INVALID_ARG, "null solution or cotangent");
        ensure_faces(ctx);
        size_t n = size_t(ctx->dev->ncells()), nf = size_t(ctx->dev->nfaces());
        for (size_t i = 0; i < n; ++i)
            if (!std::isfinite(pbar[i]) || !std::isfinite(p[i]))
                throw tpa::Error(TPA_ERR_NONFINITE, "solution and cotangent must be finite");
        if (ctx->d_face.n != nf) ctx->d_face.alloc(nf);
        cudaStream_t s = ctx->dev->stream();
        TPA_CUDA(cudaMemcpyAsync(ctx->d_x.p, p, n * sizeof(double), cudaMemcpyHostToDevice, s));
        TPA_CUDA(cudaMemcpyAsync(ctx->d_y.p, pbar, n * sizeof(double), cudaMemcpyHostToDevice, s));
        adjoint_on_device(ctx, ctx->d_x.p, ctx->d_y.p, rhs_bar ? ctx->d_y.p : nullptr,
                          kappa_bar ? ctx->d_face.p : nullptr, rtol, atol, max_cycles, precision, stats);
        if (rhs_bar) TPA_CUDA(cudaMemcpyAsync(rhs_bar, ctx->d_y.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (kappa_bar)
            TPA_CUDA(cudaMemcpyAsync(kappa_bar, ctx->d_face.p, nf * sizeof(double), cudaMemcpyDeviceToHost, s));
        TPA_CUDA(cudaStreamSynchronize(s));
    });
}

tpa_status tpa_set_stream(tpa_context* ctx, void* stream) {
    return guard(ctx, [&] {
        if (ctx->dev) TPA_CUDA(cudaStreamSynchronize(ctx->dev->stream()));
        ctx->user_stream = stream;
        if (ctx->dev) ctx->dev->set_stream(static_cast<cudaStream_t>(stream));
    });
}

tpa_status tpa_time_kernel(tpa_context* ctx, int32_t which, int32_t level, int32_t precision, int32_t iters,
                           double* ms) {
    return guard(ctx, [&] {
        if (which < 0 || which > 9 || iters <= 0 || !ms || (precision != 0 && precision != 1))
            throw tpa::Error(TPA_ERR_INVALID_ARG, "bad kernel timing request");
        ensure_device(ctx);
        *ms = ctx->dev->time_kernel(which, level, precision, iters);
    });
}

tpa_status tpa_residual_norms(tpa_context* ctx, const double* r, double out[2]) {
    return guard(ctx, [&] {
        if (!r || !out) throw tpa::Error(TPA_ERR_INVALID_ARG, "null residual or output");
        ensure_device(ctx);
        ctx->dev->residual_norms(r, out);
    });
}

tpa_status tpa_conditional_fraction_device(tpa_context* ctx, const double* fraction, double fraction_floor,
                                           double* physical, double* conditional) {
    return guard(ctx, [&] {
        if (!fraction || !conditional) throw tpa::Error(TPA_ERR_INVALID_ARG, "null argument");
        ensure_projection(ctx);
        ctx->dev->conditional_fraction(fraction, fraction_floor, physical, conditional);
    });
}

tpa_status tpa_face_coefficients_device(tpa_context* ctx, const double* conditional, double rho_liquid,
                                        double rho_gas, double* face_coefficient) {
    return guard(ctx, [&] {
        if (!conditional || !face_coefficient) throw tpa::Error(TPA_ERR_INVALID_ARG, "null argument");
        ensure_projection(ctx);
        ctx->dev->face_coefficients(conditional, rho_liquid, rho_gas, face_coefficient);
        TPA_CUDA(cudaStreamSynchronize(ctx->dev->stream()));
    });
}

tpa_status tpa_surface_tension_device(tpa_context* ctx, const double* conditional, double sigma, double curvature,
                                      int32_t formulation, double* accel_interior, double* accel_boundary) {
    return guard(ctx, [&] {
        if (!conditional || !accel_interior) throw tpa::Error(TPA_ERR_INVALID_ARG, "null argument");
        if (formulation != 0 && formulation != 1) throw tpa::Error(TPA_ERR_INVALID_ARG, "formulation must be CSF() or CGFM()");
        ensure_projection(ctx);
        ctx->dev->surface_tension(conditional, sigma, curvature, formulation, accel_interior, accel_boundary);
        TPA_CUDA(cudaStreamSynchronize(ctx->dev->stream()));
    });
}

tpa_status tpa_weighted_gradient_device(tpa_context* ctx, const double* pressure, double* grad_interior,
                                        double* grad_boundary) {
    return guard(ctx, [&] {
        if (!pressure || !grad_interior) throw tpa::Error(TPA_ERR_INVALID_ARG, "null argument");
        ensure_projection(ctx);
        ctx->dev->weighted_gradient(pressure, grad_interior, grad_boundary);
        TPA_CUDA(cudaStreamSynchronize(ctx->dev->stream()));
    });
}

tpa_status tpa_divergence_device(tpa_context* ctx, const double* u_interior, const double* u_boundary,
                                 double* divergence) {
    return guard(ctx, [&] {
        if (!u_interior || !divergence) throw tpa::Error(TPA_ERR_INVALID_ARG, "null argument");
        ensure_projection(ctx);
        if (ctx->dev->nboundary_faces() > 0 && !u_boundary)
            throw tpa::Error(TPA_ERR_INVALID_ARG, "the mesh has boundary faces: u_boundary is required");
        ctx->dev->divergence(u_interior, u_boundary, divergence);
        TPA_CUDA(cudaStreamSynchronize(ctx->dev->stream()));
    });
}

namespace {

void project_body(tpa_context* ctx, double* u_int, double* u_bnd, double* p, const tpa_projection_options* o,
                  const double* inherited, tpa_stats* stats) {
    if (!o) throw tpa::Error(TPA_ERR_INVALID_ARG, "null options");
    if (o->compatibility != 0 && o->compatibility != 1)
        throw tpa::Error(TPA_ERR_INVALID_ARG, "compatibility must be :project or :error");
    if (o->precision < 0 || o->precision > 2) throw tpa::Error(TPA_ERR_INVALID_ARG, "bad precision");
    if (o->max_cycles < 0) throw tpa::Error(TPA_ERR_INVALID_ARG, "max_cycles must be nonnegative");
    // 0 stands for "not given"; any other value (negative, inf, nan) is checked
    const double reference_dt = o->reference_dt == 0.0 ? o->dt : o->reference_dt;
    tpa::SolveStats st;
    ctx->dev->reset_launches();
    ctx->dev->project(u_int, u_bnd, p, o->dt, o->tolerance, o->max_cycles, o->compatibility, inherited,
                      reference_dt, o->precision, o->prepared != 0, st);
    TPA_CUDA(cudaStreamSynchronize(ctx->dev->stream()));
    fill_stats(st, o->precision, ctx->dev->kernel_launches(), stats);
    if (stats) {
        // `_projection_compatibility!`: dt^2 times the largest removed component mean
        const double m = st.removed_max_component_mean;
        const double scaled = (m == 0) ? 0.0 : o->dt * o->dt * m;
        stats->compatible = std::isfinite(m) && scaled <= o->tolerance;
        stats->residual_scale = 1.0 / (o->dt * o->dt);
    }
}

}  // namespace

tpa_status tpa_project_device(tpa_context* ctx, double* u_interior, double* u_boundary, double* pressure,
                              const tpa_projection_options* options, tpa_stats* stats) {
    return guard(ctx, [&] {
        if (!u_interior || !pressure) throw tpa::Error(TPA_ERR_INVALID_ARG, "null argument");
        ensure_projection(ctx);
        if (ctx->dev->nboundary_faces() > 0 && !u_boundary)
            throw tpa::Error(TPA_ERR_INVALID_ARG, "the mesh has boundary faces: u_boundary is required");
        project_body(ctx, u_interior, u_boundary, pressure, options, options ? options->inherited_divergence : nullptr,
                     stats);
    });
}

tpa_status tpa_project(tpa_context* ctx, double* u_interior, double* u_boundary, double* pressure,
                       const tpa_projection_options* options, tpa_stats* stats) {
    return guard(ctx, [&] {
        if (!u_interior || !pressure) throw tpa::Error(TPA_ERR_INVALID_ARG, "null argument");
        ensure_projection(ctx);
        const size_t n = size_t(ctx->dev->ncells()), nf = size_t(ctx->dev->nfaces()),
                     nb = size_t(ctx->dev->nboundary_faces());
        if (nb > 0 && !u_boundary) throw tpa::Error(TPA_ERR_INVALID_ARG, "the mesh has boundary faces: u_boundary is required");
        // one device buffer: u interior, u boundary, pressure, inherited divergence
        const bool inh = options && options->inherited_divergence;
        const size_t total = nf + nb + n + (inh ? n : 0);
        if (ctx->d_aux.n < total) ctx->d_aux.alloc(total);
        double* du = ctx->d_aux.p;
        double* db = du + nf;
        double* dp = db + nb;
        double* di = inh ? dp + n : nullptr;
        cudaStream_t s = ctx->dev->stream();
        TPA_CUDA(cudaMemcpyAsync(du, u_interior, nf * sizeof(double), cudaMemcpyHostToDevice, s));
        if (nb) TPA_CUDA(cudaMemcpyAsync(db, u_boundary, nb * sizeof(double), cudaMemcpyHostToDevice, s));
        TPA_CUDA(cudaMemcpyAsync(dp, pressure, n * sizeof(double), cudaMemcpyHostToDevice, s));
        if (inh) TPA_CUDA(cudaMemcpyAsync(di, options->inherited_divergence, n * sizeof(double), cudaMemcpyHostToDevice, s));
        project_body(ctx, du, db, dp, options, di, stats);
        TPA_CUDA(cudaMemcpyAsync(u_interior, du, nf * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (nb) TPA_CUDA(cudaMemcpyAsync(u_boundary, db, nb * sizeof(double), cudaMemcpyDeviceToHost, s));
        TPA_CUDA(cudaMemcpyAsync(pressure, dp, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        TPA_CUDA(cudaStreamSynchronize(s));
    });
}

tpa_status tpa_device_info(tpa_context* ctx, int64_t out[4]) {
    return guard(ctx, [&] {
        ensure_device(ctx);
        out[0] = ctx->dev->structured_levels();
        out[1] = ctx->dev->exception_rows();
        out[2] = ctx->dev->tail_first();
        out[3] = ctx->dev->fused() ? 1 : 0;
    });
}

}  // extern "C"

struct tpa_batch {
    int device = 0;
    std::string error;
    std::unique_ptr<tpa::BatchSolver> solver;
    tpa::DevArray<double> d_rhs, d_x;
};

namespace {

template <typename F>
tpa_status bguard(tpa_batch* b, F&& f) {
    if (!b) return TPA_ERR_INVALID_ARG;
    try {
        b->error.clear();
        f();
        return TPA_OK;
    } catch (const tpa::Error& e) {
        b->error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        b->error = "host allocation failed";
        return TPA_ERR_INVALID_ARG;
    } catch (const std::exception& e) {
        b->error = e.what();
        return TPA_ERR_INVALID_ARG;
    }
}

// Solves every problem; returns the first rejected problem's error (code 0: none).
tpa::Error batch_solve_body(tpa_batch* b, const double* rhs, double* x, double rtol, double atol, int32_t max_cycles,
                            int32_t compatibility, int32_t precision, tpa_stats* stats, tpa_status* statuses) {
    tpa::BatchSolver& s = *b->solver;
    std::vector<tpa::SolveStats> st;
    std::vector<int> status;
    std::vector<std::string> msg;
    s.reset_launches();
    s.solve(rhs, x, rtol, atol, max_cycles, compatibility, precision, st, status, msg);
    for (int k = 0; k < s.count(); ++k) {
        if (stats) fill_stats(st[size_t(k)], precision, s.kernel_launches(), stats + k);
        if (statuses) statuses[k] = status[size_t(k)];
    }
    for (int k = 0; k < s.count(); ++k)
        if (status[size_t(k)]) return tpa::Error(status[size_t(k)], "problem " + std::to_string(k) + ": " + msg[size_t(k)]);
    return tpa::Error(0, "");
}

}  // namespace

extern "C" {

tpa_status tpa_batch_create(tpa_batch** out, tpa_context* const* ctxs, int32_t count) {
    if (!out || count <= 0 || !ctxs) return TPA_ERR_INVALID_ARG;
    *out = nullptr;
    tpa_batch* b = nullptr;
    try {
        b = new tpa_batch();
    } catch (...) {
        return TPA_ERR_INVALID_ARG;
    }
    tpa_status st = bguard(b, [&] {
        std::vector<const tpa::Hierarchy*> hs;
        for (int32_t k = 0; k < count; ++k) {
            if (!ctxs[k]) throw tpa::Error(TPA_ERR_INVALID_ARG, "null context");
            if (!ctxs[k]->have_hierarchy)
                throw tpa::Error(TPA_ERR_STATE, "problem " + std::to_string(k) + " has no hierarchy");
            if (ctxs[k]->device != ctxs[0]->device) throw tpa::Error(TPA_ERR_INVALID_ARG, "contexts on different devices");
            ensure_host_fresh(ctxs[k]);
            if (ctxs[k]->hier.opts.smoother != 0)
                throw tpa::Error(TPA_ERR_UNSUPPORTED, "the merged batch smooths with damped Jacobi only");
            if (ctxs[k]->hier.levels[0].op.any_open())
                throw tpa::Error(TPA_ERR_UNSUPPORTED, "the merged batch takes closed sides only (no open pressure sides)");
            hs.push_back(&ctxs[k]->hier);
        }
        int devices = 0;
        if (cudaGetDeviceCount(&devices) != cudaSuccess || devices <= ctxs[0]->device)
            throw tpa::Error(TPA_ERR_CUDA, "no usable CUDA device for the B200 solver");
        b->device = ctxs[0]->device;
        b->solver.reset(new tpa::BatchSolver(b->device, hs));
    });
    if (st != TPA_OK) {
        // keep the handle so that the caller can read the message, then destroy it
        *out = b;
        return st;
    }
    *out = b;
    return TPA_OK;
}

void tpa_batch_destroy(tpa_batch* b) {
    if (!b) return;
    try {
        b->d_rhs.free();
        b->d_x.free();
        b->solver.reset();
    } catch (...) {
    }
    delete b;
}

const char* tpa_batch_last_error(const tpa_batch* b) { return b ? b->error.c_str() : "null batch"; }

tpa_status tpa_batch_sizes(const tpa_batch* cb, int64_t out[4]) {
    auto* b = const_cast<tpa_batch*>(cb);
    return bguard(b, [&] {
        if (!b->solver) throw tpa::Error(TPA_ERR_STATE, "batch was not built");
        out[0] = b->solver->count();
        out[1] = b->solver->fine_cells();
        out[2] = b->solver->levels();
        out[3] = b->solver->tail_levels();
    });
}

tpa_status tpa_batch_offsets(const tpa_batch* cb, int64_t* offsets) {
    auto* b = const_cast<tpa_batch*>(cb);
    return bguard(b, [&] {
        if (!b->solver) throw tpa::Error(TPA_ERR_STATE, "batch was not built");
        const auto& F = b->solver->offsets();
        std::memcpy(offsets, F.data(), F.size() * sizeof(int64_t));
    });
}

tpa_status tpa_batch_set_stream(tpa_batch* b, void* stream) {
    return bguard(b, [&] {
        if (!b->solver) throw tpa::Error(TPA_ERR_STATE, "batch was not built");
        TPA_CUDA(cudaStreamSynchronize(b->solver->stream()));
        b->solver->set_stream(static_cast<cudaStream_t>(stream));
    });
}

tpa_status tpa_batch_solve_device(tpa_batch* b, const double* rhs, double* x, double rtol, double atol,
                                  int32_t max_cycles, int32_t compatibility, int32_t precision, tpa_stats* stats,
                                  tpa_status* statuses) {
    return bguard(b, [&] {
        if (!b->solver) throw tpa::Error(TPA_ERR_STATE, "batch was not built");
        if (!rhs || !x) throw tpa::Error(TPA_ERR_INVALID_ARG, "null rhs or solution");
        tpa::Error e = batch_solve_body(b, rhs, x, rtol, atol, max_cycles, compatibility, precision, stats, statuses);
        if (e.code) throw e;
    });
}

tpa_status tpa_batch_solve(tpa_batch* b, const double* rhs, double* x, double rtol, double atol, int32_t max_cycles,
                           int32_t compatibility, int32_t precision, tpa_stats* stats, tpa_status* statuses) {
    return bguard(b, [&] {
        if (!b->solver) throw tpa::Error(TPA_ERR_STATE, "batch was not built");
        if (!rhs || !x) throw tpa::Error(TPA_ERR_INVALID_ARG, "null rhs or solution");
        const size_t n = size_t(b->solver->fine_cells());
        for (size_t i = 0; i < n; ++i)
            if (!std::isfinite(rhs[i])) throw tpa::Error(TPA_ERR_NONFINITE, "right-hand side must be finite");
        if (b->d_rhs.n != n) b->d_rhs.alloc(n);
        if (b->d_x.n != n) b->d_x.alloc(n);
        cudaStream_t s = b->solver->stream();
        TPA_CUDA(cudaSetDevice(b->device));
        TPA_CUDA(cudaMemcpyAsync(b->d_rhs.p, rhs, n * sizeof(double), cudaMemcpyHostToDevice, s));
        TPA_CUDA(cudaMemcpyAsync(b->d_x.p, x, n * sizeof(double), cudaMemcpyHostToDevice, s));
        tpa::Error e = batch_solve_body(b, b->d_rhs.p, b->d_x.p, rtol, atol, max_cycles, compatibility, precision,
                                        stats, statuses);
        TPA_CUDA(cudaMemcpyAsync(x, b->d_x.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        TPA_CUDA(cudaStreamSynchronize(s));
        if (e.code) throw e;
    });
}

}  // extern "C"

namespace {
tpa::TuneConfig from_c(const tpa_tune_config& c) {
    tpa::TuneConfig t;
    t.tail_cells = c.tail_cells;
    t.tail_ctas = c.tail_ctas;
    t.structured = c.structured;
    t.vectorized = c.vectorized;
    t.pdl = c.pdl;
    t.fuse_restrict = c.fuse_restrict;
    t.persistent = c.persistent;
    t.tiles = c.tiles;
    return t;
}
tpa_tune_config to_c(const tpa::TuneConfig& t, double ms) {
    tpa_tune_config c;
    c.tail_cells = t.tail_cells;
    c.tail_ctas = t.tail_ctas;
    c.structured = t.structured;
    c.vectorized = t.vectorized;
    c.pdl = t.pdl;
    c.fuse_restrict = t.fuse_restrict;
    c.persistent = t.persistent;
    c.tiles = t.tiles;
    c.ms_per_vcycle = ms;
    return c;
}
}  // namespace

extern "C" {

tpa_status tpa_autotune(tpa_context* ctx, int32_t precision, int32_t vcycles, tpa_tune_config* best,
                        tpa_tune_config* tried, int32_t capacity, int32_t* ntried) {
    return guard(ctx, [&] {
        if (precision < 0 || precision > 2) throw tpa::Error(TPA_ERR_INVALID_ARG, "bad precision");
        if (vcycles <= 0) throw tpa::Error(TPA_ERR_INVALID_ARG, "vcycles must be positive");
        precision = std::min(precision, 1);  // the refinement solve runs the FP32 V-cycle
        ensure_device(ctx);
        ensure_host_fresh(ctx);  // stencil copies come from the host levels
        tpa::DeviceSolver& d = *ctx->dev;
        std::vector<tpa::TuneConfig> cand;
        for (int cells : {1024, 2048, 4096, 8192})
            for (int ctas : {1, 4})
                for (int st : {1, 2}) {
                    tpa::TuneConfig c;
                    c.tail_cells = cells;
                    c.tail_ctas = ctas;
                    c.structured = st;
                    c.vectorized = 1;
                    c.pdl = 1;
                    c.fuse_restrict = 0;
                    c.persistent = 0;
                    c.tiles = 0;
                    cand.push_back(c);
                }
        std::vector<std::pair<tpa::TuneConfig, double>> res;
        auto run = [&](const tpa::TuneConfig& c) {
            d.reconfigure(ctx->hier, c);
            res.emplace_back(d.effective_tuning(), d.time_vcycles(precision, vcycles));
        };
        for (const auto& c : cand) run(c);
        auto best_of = [&] {
            size_t b = 0;
            for (size_t k = 1; k < res.size(); ++k)
                if (res[k].second < res[b].second) b = k;
            return b;
        };
        // then the best one without the vectorized kernels and without PDL
        tpa::TuneConfig b0 = res[best_of()].first;
        tpa::TuneConfig nv = b0, np = b0;
        nv.vectorized = 0;
        np.pdl = 0;
        tpa::TuneConfig fr = b0, pe = b0;
        fr.fuse_restrict = 1;
        tpa::TuneConfig fr_small = b0, fr_mid = b0;  // fused on the small levels only
        fr_small.fuse_restrict = 16384;
        fr_mid.fuse_restrict = 65536;
        pe.persistent = 1;
        pe.tail_ctas = 1;
        run(nv);
        run(np);
        run(fr);
        run(fr_small);
        run(fr_mid);
        run(pe);
        // the CSR levels on haloed block tiles (two launches per level), with
        // the tail sizes around the best one
        for (int tiles : {1, 2, 3})
            for (int cells : {256, 1024, 2048, 4096}) {
                tpa::TuneConfig tl = b0;
                tl.tiles = tiles;
                tl.tail_cells = cells;
                run(tl);
            }
        // the periodic lattice levels on the row-streaming kernels: the larger
        // ones (4) or all (5), with the small tails (the streamed levels reach
        // down to 32 x 32 cells)
        for (int tiles : {4, 5})
            for (int cells : {256, 1024, 2048}) {
                tpa::TuneConfig tl = b0;
                tl.tiles = tiles;
                tl.tail_cells = cells;
                run(tl);
            }
        const size_t b = best_of();
        d.reconfigure(ctx->hier, res[b].first);
        if (best) *best = to_c(res[b].first, res[b].second);
        if (ntried) *ntried = int32_t(res.size());
        for (int32_t k = 0; tried && k < capacity && size_t(k) < res.size(); ++k)
            tried[k] = to_c(res[size_t(k)].first, res[size_t(k)].second);
    });
}

tpa_status tpa_set_tuning(tpa_context* ctx, const tpa_tune_config* cfg) {
    return guard(ctx, [&] {
        if (!cfg) throw tpa::Error(TPA_ERR_INVALID_ARG, "null configuration");
        if (cfg->tail_ctas > 8 || cfg->structured > 2 || cfg->tiles > 5)
            throw tpa::Error(TPA_ERR_INVALID_ARG, "bad configuration");
        ensure_device(ctx);
        ensure_host_fresh(ctx);  // stencil copies come from the host levels
        ctx->dev->reconfigure(ctx->hier, from_c(*cfg));
    });
}

tpa_status tpa_tiled_levels(tpa_context* ctx, int32_t* count) {
    return guard(ctx, [&] {
        if (!count) throw tpa::Error(TPA_ERR_INVALID_ARG, "null output");
        ensure_device(ctx);
        *count = ctx->dev->tiled_levels();
    });
}

tpa_status tpa_streamed_levels(tpa_context* ctx, int32_t* count) {
    return guard(ctx, [&] {
        if (!count) throw tpa::Error(TPA_ERR_INVALID_ARG, "null output");
        ensure_device(ctx);
        *count = ctx->dev->streamed_levels();
    });
}

tpa_status tpa_get_tuning(tpa_context* ctx, tpa_tune_config* cfg) {
    return guard(ctx, [&] {
        if (!cfg) throw tpa::Error(TPA_ERR_INVALID_ARG, "null configuration");
        ensure_device(ctx);
        *cfg = to_c(ctx->dev->effective_tuning(), 0.0);
    });
}

}  // extern "C"

extern "C" {

tpa_status tpa_synchronize(tpa_context* ctx) {
    return guard(ctx, [&] {
        if (ctx->dev) TPA_CUDA(cudaStreamSynchronize(ctx->dev->stream()));
    });
}

}  // extern "C"

// ---------------------------------------------------------------- CMDGFM

namespace {

// CSR rows from the C-ABI arrays, checked: row pointers from 0, nondecreasing,
// columns in [0, ncol) and increasing within a row, finite values
tpa::CsrRows csr_from(int64_t nrow, int64_t ncol, const int64_t* ptr, const int32_t* col, const double* val,
                      const char* what) {
    tpa::CsrRows m;
    m.n = nrow;
    if (nrow == 0) {
        m.ptr.assign(1, 0);
        return m;
    }
    if (!ptr || (ptr[nrow] > 0 && (!col || !val)))
        throw tpa::Error(TPA_ERR_INVALID_ARG, std::string(what) + ": null array");
    if (ptr[0] != 0) throw tpa::Error(TPA_ERR_INVALID_ARG, std::string(what) + ": row_ptr[0] must be 0");
    m.ptr.assign(ptr, ptr + nrow + 1);
    for (int64_t r = 0; r < nrow; ++r) {
        if (ptr[r + 1] < ptr[r]) throw tpa::Error(TPA_ERR_INVALID_ARG, std::string(what) + ": decreasing row_ptr");
        for (int64_t k = ptr[r]; k < ptr[r + 1]; ++k) {
            if (col[k] < 0 || col[k] >= ncol)
                throw tpa::Error(TPA_ERR_INVALID_ARG, std::string(what) + ": column out of range");
            if (k > ptr[r] && col[k] <= col[k - 1])
                throw tpa::Error(TPA_ERR_INVALID_ARG, std::string(what) + ": columns not increasing within a row");
            if (!std::isfinite(val[k])) throw tpa::Error(TPA_ERR_NONFINITE, std::string(what) + ": non-finite entry");
        }
    }
    m.col.assign(col, col + ptr[nrow]);
    m.val.assign(val, val + ptr[nrow]);
    return m;
}

template <typename T>
std::vector<T> host_vector(const T* p, int64_t n, const char* what) {
    if (n > 0 && !p) throw tpa::Error(TPA_ERR_INVALID_ARG, std::string("null ") + what);
    return n > 0 ? std::vector<T>(p, p + n) : std::vector<T>();
}

// the system as the library takes it, every argument checked; ncells < 0
// skips the cell-range check (no context)
tpa::CmdgfmInput cmdgfm_input(const tpa_cmdgfm_system* sys, int64_t ncells) {
    if (!sys) throw tpa::Error(TPA_ERR_INVALID_ARG, "null system");
    if (sys->np < 0 || sys->nx < 0 || sys->na < 0) throw tpa::Error(TPA_ERR_INVALID_ARG, "negative size");
    const int64_t n = sys->np + sys->nx;
    if (n >= (int64_t(1) << 31)) throw tpa::Error(TPA_ERR_INVALID_ARG, "the system has 2^31 or more unknowns");
    tpa::CmdgfmInput in;
    in.np = sys->np;
    in.m = csr_from(n, n, sys->row_ptr, sys->col, sys->val, "system");
    in.rhs = host_vector(sys->rhs, n, "rhs");
    in.cell = host_vector(sys->pressure_cell, sys->np, "pressure_cell");
    in.anchor = host_vector(sys->pressure_anchor, sys->np, "pressure_anchor");
    in.weight = host_vector(sys->defect_weight, n, "defect_weight");
    in.extra = csr_from(sys->na, n, sys->extra_row_ptr, sys->extra_col, sys->extra_val, "anchor rows");
    in.extra_rhs = host_vector(sys->extra_rhs, sys->na, "extra_rhs");
    in.extra_weight = host_vector(sys->extra_weight, sys->na, "extra_weight");
    in.row_scale = host_vector(sys->row_scale, n, "row_scale");
    in.col_scale = host_vector(sys->col_scale, n, "col_scale");
    for (int64_t i = 0; i < sys->np; ++i) {
        const int32_t c = in.cell[size_t(i)], a = in.anchor[size_t(i)];
        if (c < 0 || a < 0 || (ncells >= 0 && (c >= ncells || a >= ncells)))
            throw tpa::Error(TPA_ERR_INVALID_ARG, "pressure cell or anchor out of the mesh");
        if (c == a) throw tpa::Error(TPA_ERR_INVALID_ARG, "a retained cell is its own anchor");
    }
    for (double v : in.rhs)
        if (!std::isfinite(v)) throw tpa::Error(TPA_ERR_NONFINITE, "right-hand side must be finite");
    for (const auto* w : {&in.weight, &in.extra_weight})
        for (double v : *w)
            if (!(v >= 0 && std::isfinite(v))) throw tpa::Error(TPA_ERR_INVALID_ARG, "defect weights must be finite and nonnegative");
    for (double v : in.extra_rhs)
        if (!std::isfinite(v)) throw tpa::Error(TPA_ERR_NONFINITE, "anchor right-hand side must be finite");
    for (const auto* w : {&in.row_scale, &in.col_scale})
        for (double v : *w)
            if (!(v > 0 && std::isfinite(v))) throw tpa::Error(TPA_ERR_INVALID_ARG, "scalings must be finite and positive");
    if (!(sys->drop_tolerance >= 0 && std::isfinite(sys->drop_tolerance)))
        throw tpa::Error(TPA_ERR_INVALID_ARG, "drop_tolerance must be nonnegative");
    if (!(sys->tolerance > 0 && std::isfinite(sys->tolerance)))
        throw tpa::Error(TPA_ERR_INVALID_ARG, "tolerance must be strictly positive");
    if (sys->max_iterations <= 0) throw tpa::Error(TPA_ERR_INVALID_ARG, "max_iterations must be strictly positive");
    if (sys->precision != 0 && sys->precision != 1) throw tpa::Error(TPA_ERR_INVALID_ARG, "bad precision");
    in.tolerance = sys->tolerance;
    in.max_iterations = sys->max_iterations;
    in.precision = sys->precision;
    if (sys->warm_start != 0 && sys->warm_start != 1) throw tpa::Error(TPA_ERR_INVALID_ARG, "warm_start must be 0 or 1");
    in.warm_start = sys->warm_start != 0;
    if (sys->initial_pressure) in.initial.assign(sys->initial_pressure, sys->initial_pressure + sys->np);
    return in;
}

void copy_csr(const tpa::CsrRows& m, int64_t* nnz, int64_t* ptr, int32_t* col, double* val) {
    if (nnz) *nnz = int64_t(m.col.size());
    if (ptr) std::memcpy(ptr, m.ptr.data(), m.ptr.size() * sizeof(int64_t));
    if (col) std::memcpy(col, m.col.data(), m.col.size() * sizeof(int32_t));
    if (val) std::memcpy(val, m.val.data(), m.val.size() * sizeof(double));
}

}  // namespace

tpa_status tpa_cmdgfm_solve(tpa_context* ctx, const tpa_cmdgfm_system* system, double* solution,
                            tpa_cmdgfm_stats* stats) {
    return guard(ctx, [&] {
        if (!solution && system && system->np + system->nx > 0)
            throw tpa::Error(TPA_ERR_INVALID_ARG, "null solution");
        ensure_device(ctx);
        const tpa::CmdgfmInput in = cmdgfm_input(system, ctx->dev->ncells());
        const auto t0 = std::chrono::steady_clock::now();
        const tpa::CmdgfmFactor f = tpa::cmdgfm_factor(in.m, in.np, system->drop_tolerance);
        const double setup_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (!ctx->cmdgfm) ctx->cmdgfm.reset(new tpa::CmdgfmDevice());
        tpa::CmdgfmStats st;
        ctx->cmdgfm->solve(*ctx->dev, in, f, solution, st);
        if (stats) {
            std::memset(stats, 0, sizeof(*stats));
            stats->converged = st.converged ? 1 : 0;
            stats->iterations = st.iterations;
            stats->attempts = st.attempts;
            stats->kernel_launches = st.launches;
            stats->initial_residual = st.initial_residual;
            stats->final_residual = st.final_residual;
            stats->pressure_defect = st.pressure_defect;
            stats->jump_defect = st.jump_defect;
            stats->anchor_defect = st.anchor_defect;
            stats->setup_ms = setup_ms;
            stats->device_ms = st.device_ms;
            stats->factor_entries = int64_t(f.lower.col.size() + f.upper.col.size() + f.pivot.size());
            stats->lower_levels = f.nx ? f.lsched.levels() : 0;
            stats->upper_levels = f.nx ? f.usched.levels() : 0;
            stats->inverse_entries = st.inverse ? int64_t(f.linv.col.size() + f.uinv.col.size()) : 0;
            stats->initial_guess_used = st.initial_guess_used ? 1 : 0;
        }
    });
}

tpa_status tpa_cmdgfm_factor(const tpa_cmdgfm_system* system, int64_t* s_nnz, int64_t* s_ptr, int32_t* s_col,
                             double* s_val, int64_t* l_nnz, int64_t* l_ptr, int32_t* l_col, double* l_val,
                             int64_t* u_nnz, int64_t* u_ptr, int32_t* u_col, double* u_val) {
    try {
        const tpa::CmdgfmInput in = cmdgfm_input(system, -1);
        const tpa::CmdgfmFactor f = tpa::cmdgfm_factor(in.m, in.np, system->drop_tolerance);
        copy_csr(f.schur, s_nnz, s_ptr, s_col, s_val);
        copy_csr(f.lower, l_nnz, l_ptr, l_col, l_val);
        // U with its pivot first in each row, the rest in column order
        tpa::CsrRows u;
        u.n = f.upper.n;
        u.ptr.assign(1, 0);
        for (int64_t r = 0; r < f.upper.n; ++r) {
            u.col.push_back(int32_t(r));
            u.val.push_back(f.pivot[size_t(r)]);
            for (int64_t k = f.upper.ptr[size_t(r)]; k < f.upper.ptr[size_t(r) + 1]; ++k) {
                u.col.push_back(f.upper.col[size_t(k)]);
                u.val.push_back(f.upper.val[size_t(k)]);
            }
            u.ptr.push_back(int64_t(u.col.size()));
        }
        copy_csr(u, u_nnz, u_ptr, u_col, u_val);
        return TPA_OK;
    } catch (const tpa::Error& e) {
        return e.code;
    } catch (const std::exception&) {
        return TPA_ERR_INVALID_ARG;
    }
}
