// Merged batch of independent pressure solves (batch.cuh): host assembly of
// the batch levels from the problems' hierarchies, the per-problem FP64 CG
// kernels, and the solve driver (one graph launch per Krylov run of the whole
// batch).  Each problem follows `solve!` (src/solvers/multigrid/
// elliptic_solver.jl:628-675 of ronaldremmerswaal/TwoPhaseAMR.jl): b = V f,
// component projection, CG with the strong-residual callback, restarts from the
// true residual (`_run_krylov_reliably!`, :487-526) and the final gauge.
#include "batch.hpp"

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstring>

namespace tpa {
namespace {

enum BCounter { bcRestrict, bcPost, bcAp, bcUpdMax, bcUpdSum, bcZ, bcSum, bcMax, bcCount };

// ---- fine-space FP64 kernels (one BFItem per CTA) --------------------------------

struct FineCsr {
    const int* rp;
    const int* ci;
    const double* val;
    const double* vol;
};

__device__ __forceinline__ double frow(const FineCsr& A, const double* v, int i) {
    double acc = 0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) acc += A.val[k] * v[A.ci[k]];
    return acc;
}

// A x as sum_j a_ij (x_j - x_i) for the true residual: the rows sum to zero, and
// this form rounds at the level of the face fluxes (x_j - x_i), as the
// factorized action does, rather than at that of a_ii x_i
__device__ __forceinline__ double frow_diff(const FineCsr& A, const double* v, int i) {
    const double vi = v[i];
    double acc = 0;
    for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) acc += A.val[k] * (v[A.ci[k]] - vi);
    return acc;
}

// b = V f and x = x0 (zero where V = 0)
__global__ void bk_prepare(const BFItem* __restrict__ fi, FineCsr A, const double* __restrict__ rhs,
                           const double* __restrict__ x0, double* __restrict__ b, double* __restrict__ x) {
    const BFItem it = fi[blockIdx.x];
    const int i = it.begin + int(threadIdx.x);
    if (i >= it.end) return;
    const double V = A.vol[i];
    b[i] = V > 0 ? rhs[i] * V : 0.0;
    x[i] = V > 0 ? x0[i] : 0.0;
}

// per-problem sum of w .* v (w null: of v; absval: of |v|) for the problems with sel[k]
__global__ void bk_sum(const BFItem* __restrict__ fi, const int* __restrict__ pfirst, const int* __restrict__ pcount,
                       const double* __restrict__ v, const double* __restrict__ w, int absval, double* partial,
                       unsigned* counters, double* __restrict__ out) {
    const BFItem it = fi[blockIdx.x];
    const int i = it.begin + int(threadIdx.x);
    double a = 0;
    if (i < it.end) {
        a = w ? w[i] * v[i] : v[i];
        if (absval) a = fabs(a);
    }
    double total;
    if (fold_problem(a, partial, counters + it.prob, pfirst[it.prob], pcount[it.prob], total) && threadIdx.x == 0)
        out[it.prob] = total;
}

// v -= (w ? w : 1) * coef[prob]
__global__ void bk_sub(const BFItem* __restrict__ fi, double* __restrict__ v, const double* __restrict__ w,
                       const double* __restrict__ coef) {
    const BFItem it = fi[blockIdx.x];
    const double c = coef[it.prob];
    if (c == 0) return;
    const int i = it.begin + int(threadIdx.x);
    if (i < it.end) v[i] -= (w ? w[i] : 1.0) * c;
}

// r = b - A x (problems with sel[k], or all); per problem: max |r|/V into
// out_max (fold 1), and sum V (r/V)^2 into out_l2 or sum r into st->rsum (fold 2)
__global__ void bk_residual64(const BFItem* __restrict__ fi, const int* __restrict__ pfirst,
                              const int* __restrict__ pcount, FineCsr A, const double* __restrict__ b,
                              const double* __restrict__ x, double* __restrict__ r, double* p1, double* p2,
                              unsigned* c1, unsigned* c2, double* __restrict__ out_max, double* __restrict__ out_l2,
                              BState* st, const int* __restrict__ sel) {
    pdl_entry();
    const BFItem it = fi[blockIdx.x];
    if (sel && !sel[it.prob]) return;
    const int i = it.begin + int(threadIdx.x);
    double q = 0, l2 = 0, sum = 0;
    if (i < it.end) {
        const double ri = b[i] - frow_diff(A, x, i);
        r[i] = ri;
        const double V = A.vol[i];
        if (V > 0) {
            q = fabs(ri) / V;
            if (ri != ri) q = NAN;
            l2 = ri * ri / V;
        }
        sum = ri;
    }
    const int f = pfirst[it.prob], c = pcount[it.prob];
    double total;
    if (out_max && fold_problem_max(q, p1, c1 + it.prob, f, c, total) && threadIdx.x == 0) out_max[it.prob] = total;
    if (out_l2 && fold_problem(l2, p2, c2 + it.prob, f, c, total) && threadIdx.x == 0) out_l2[it.prob] = total;
    if (st && fold_problem(sum, p2, c2 + it.prob, f, c, total) && threadIdx.x == 0) st[it.prob].rsum = total;
}

// per problem: max over cells of (|A||x|)_i / V_i and |b_i| / V_i (the roundoff floor inputs)
__global__ void bk_abs_bound(const BFItem* __restrict__ fi, const int* __restrict__ pfirst,
                             const int* __restrict__ pcount, FineCsr A, const double* __restrict__ b,
                             const double* __restrict__ x, double* partial, unsigned* counters,
                             double* __restrict__ out) {
    const BFItem it = fi[blockIdx.x];
    const int i = it.begin + int(threadIdx.x);
    double q = 0;
    if (i < it.end) {
        const double V = A.vol[i];
        if (V > 0) {
            double acc = 0;
            for (int k = A.rp[i]; k < A.rp[i + 1]; ++k) acc += fabs(A.val[k]) * fabs(x[A.ci[k]]);
            q = fmax(acc / V, fabs(b[i]) / V);
        }
    }
    double total;
    if (fold_problem_max(q, partial, counters + it.prob, pfirst[it.prob], pcount[it.prob], total) &&
        threadIdx.x == 0)
        out[it.prob] = total;
}

__device__ __forceinline__ void balpha(double pAp, BState* s) {
    const double eps = 2.220446049250313e-16;
    s->pAp = pAp;
    if (pAp <= eps * s->pnorm2 && fabs(pAp) <= eps * s->pnorm2) {
        s->flags |= 2;
        s->alpha = 0;
    } else {
        s->alpha = s->gamma / pAp;
    }
}

__global__ void bk_cg_ap(const BFItem* __restrict__ fi, const int* __restrict__ pfirst,
                         const int* __restrict__ pcount, FineCsr A, const double* __restrict__ p,
                         double* __restrict__ ap, double* partial, unsigned* counters, BState* st,
                         const int* __restrict__ active) {
    pdl_entry();
    const BFItem it = fi[blockIdx.x];
    if (!active[it.prob]) return;
    const int i = it.begin + int(threadIdx.x);
    double v = 0;
    if (i < it.end) {
        const double y = frow(A, p, i);
        ap[i] = y;
        v = p[i] * y;
    }
    double total;
    if (fold_problem(v, partial, counters + it.prob, pfirst[it.prob], pcount[it.prob], total) && threadIdx.x == 0)
        balpha(total, st + it.prob);
}

__global__ void bk_cg_update(const BFItem* __restrict__ fi, const int* __restrict__ pfirst,
                             const int* __restrict__ pcount, const double* __restrict__ vol, double* __restrict__ x,
                             double* __restrict__ r, const double* __restrict__ p, const double* __restrict__ ap,
                             double* pmax, double* psum, unsigned* cmax, unsigned* csum, BState* st,
                             const int* __restrict__ active) {
    pdl_entry();
    const BFItem it = fi[blockIdx.x];
    if (!active[it.prob]) return;
    const BState& s = st[it.prob];
    const bool skip = s.flags & 2;
    const double alpha = s.alpha;
    const int i = it.begin + int(threadIdx.x);
    double q = 0, sum = 0;
    if (i < it.end) {
        double ri = r[i];
        if (!skip) {
            x[i] += alpha * p[i];
            ri -= alpha * ap[i];
            r[i] = ri;
        }
        const double V = vol[i];
        if (V > 0) {
            q = fabs(ri) / V;
            if (q != q) q = NAN;
        }
        sum = ri;
    }
    const int f = pfirst[it.prob], c = pcount[it.prob];
    double total;
    if (fold_problem_max(q, pmax, cmax + it.prob, f, c, total) && threadIdx.x == 0) st[it.prob].strong_max = total;
    if (fold_problem(sum, psum, csum + it.prob, f, c, total) && threadIdx.x == 0) st[it.prob].rsum = total;
}

// z = V-cycle output minus its mean; gamma = r'z; the stopping rules per problem
template <typename T>
__global__ void bk_cg_z(const BFItem* __restrict__ fi, const int* __restrict__ pfirst, const int* __restrict__ pcount,
                        const BLevel<T>* __restrict__ lv, const double* __restrict__ mean,
                        const double* __restrict__ r, double* __restrict__ z, double* __restrict__ p, double* partial,
                        unsigned* counters, BState* st, int* active, int init) {
    pdl_entry();
    const BFItem it = fi[blockIdx.x];
    if (!active[it.prob]) return;
    const double m = mean[it.prob];
    const T* xv = lv[it.lvl].x;
    const int i = it.begin + int(threadIdx.x);
    double v = 0;
    if (i < it.end) {
        const double zi = double(xv[i + it.off]) - m;
        z[i] = zi;
        if (init) p[i] = zi;
        v = r[i] * zi;
    }
    double g;
    if (!fold_problem(v, partial, counters + it.prob, pfirst[it.prob], pcount[it.prob], g) || threadIdx.x != 0)
        return;
    BState* s = st + it.prob;
    bool stop;
    if (init) {
        s->gamma = g;
        s->pnorm2 = g;
        s->rnorm = sqrt(g);
        s->beta = 0;
        s->iter = 0;
        s->flags = g == 0 ? 8 : 0;
        stop = g == 0 || s->itmax <= 0;
    } else if (s->flags & 2) {
        stop = true;
    } else {
        const double rnorm = sqrt(g);
        s->rnorm = rnorm;
        const bool solved = rnorm + 1.0 <= 1.0;
        if (!solved) {
            const double beta = g / s->gamma;
            s->beta = beta;
            s->pnorm2 = g + beta * beta * s->pnorm2;
            s->gamma = g;
        } else {
            s->flags |= 4;
        }
        s->iter += 1;
        if (s->strong_max <= s->target) s->flags |= 1;
        stop = solved || s->iter >= s->itmax || (s->flags & 1);
    }
    if (stop) active[it.prob] = 0;
}

__global__ void bk_cg_p(const BFItem* __restrict__ fi, double* __restrict__ p, const double* __restrict__ z,
                        const BState* __restrict__ st, const int* __restrict__ active) {
    pdl_entry();
    const BFItem it = fi[blockIdx.x];
    if (!active[it.prob]) return;
    const BState& s = st[it.prob];
    if (s.flags & 6) return;
    const int i = it.begin + int(threadIdx.x);
    if (i < it.end) p[i] = z[i] + s.beta * p[i];
}

// loop condition of the graph: any problem still iterating
__global__ void bk_cg_cond(const int* __restrict__ active, int count, cudaGraphConditionalHandle handle) {
    pdl_entry();
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int k = threadIdx.x; k < count; k += blockDim.x)
        if (active[k]) any = 1;
    __syncthreads();
    if (threadIdx.x == 0) cudaGraphSetConditional(handle, any ? 1u : 0u);
}

__global__ void bk_state_init(BState* st, const double* __restrict__ target, const int* __restrict__ itmax,
                              int count) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    st[k].target = target[k];
    st[k].itmax = itmax[k];
    st[k].flags = 0;
    st[k].iter = 0;
}

__global__ void bk_copy_out(const BFItem* __restrict__ fi, const double* __restrict__ src, double* __restrict__ dst) {
    const BFItem it = fi[blockIdx.x];
    const int i = it.begin + int(threadIdx.x);
    if (i < it.end) dst[i] = src[i];
}

struct Launch {
    cudaStream_t s;
    bool pdl;
    template <typename... KArgs, typename... Args>
    void operator()(void (*kernel)(KArgs...), int grid, int block, size_t smem, Args... args) const {
        if (grid <= 0) return;
        cudaLaunchConfig_t cfg;
        std::memset(&cfg, 0, sizeof(cfg));
        cfg.gridDim = dim3(unsigned(grid));
        cfg.blockDim = dim3(unsigned(block));
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = at;
        cfg.numAttrs = pdl ? 1 : 0;
        TPA_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
    }
};

template <typename T>
std::vector<T> cast_vec(const std::vector<double>& v) {
    return std::vector<T>(v.begin(), v.end());
}

}  // namespace

// ---------------------------------------------------------------------------------

BatchSolver::BatchSolver(int device, const std::vector<const Hierarchy*>& hs) : device_(device) {
    TPA_CUDA(cudaSetDevice(device_));
    TPA_CUDA(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking));
    stream_ = own_stream_;
    build(hs);
}

BatchSolver::~BatchSolver() {
    cudaSetDevice(device_);
    for (auto& e : exec_)
        if (e) cudaGraphExecDestroy(e);
    if (own_stream_) cudaStreamDestroy(own_stream_);
}

void BatchSolver::build(const std::vector<const Hierarchy*>& hs) {
    const int K = int(hs.size());
    if (K <= 0) throw Error(1, "a batch needs at least one problem");
    K_ = K;
    int Lmax = 0;
    for (const Hierarchy* h : hs) {
        if (!h || h->levels.empty()) throw Error(7, "every problem needs a hierarchy");
        if (h->levels.size() < 2) throw Error(5, "the batched solve needs at least two levels per problem");
        if (h->coarse_n != h->levels.back().op.A.n ||
            h->coarse_inverse.size() != size_t(h->coarse_n) * size_t(h->coarse_n))
            throw Error(7, "coarsest-level inverse does not match the coarsest level");
        if (h->opts.pre_sweeps != 2 || h->opts.post_sweeps != 2)
            throw Error(5, "the batched solve runs the default cycle (two pre- and two post-sweeps)");
        for (const HostLevel& l : h->levels)
            if (l.op.singular && l.op.comp.volume.size() > 1)
                throw Error(5, "the batched solve supports one ungauged component per level");
        Lmax = std::max(Lmax, int(h->levels.size()));
    }
    L_ = Lmax;
    // tail: the last T batch levels, every problem's share of each at most
    // kBatchTailCells cells, and no problem's finest level among them
    int T = std::min(kBatchTailLevels, Lmax);
    for (const Hierarchy* h : hs) {
        const int Lk = int(h->levels.size());
        int t = 0;
        while (t < Lk - 1 && t < kBatchTailLevels && h->levels[size_t(Lk - 1 - t)].op.A.n <= kBatchTailCells) ++t;
        T = std::min(T, std::max(t, 1));
        if (Lk < 2) T = 1;
    }
    for (const Hierarchy* h : hs)
        if (int(h->levels.size()) <= T && T > 1) T = 1;
    T_ = T;
    // row offsets per level and problem
    std::vector<std::vector<int64_t>> M(size_t(Lmax), std::vector<int64_t>(size_t(K), -1));
    std::vector<int64_t> nlev(size_t(Lmax), 0);
    for (int j = 0; j < Lmax; ++j)
        for (int k = 0; k < K; ++k) {
            const int Lk = int(hs[size_t(k)]->levels.size());
            const int l = j - (Lmax - Lk);
            if (l < 0) continue;
            M[size_t(j)][size_t(k)] = nlev[size_t(j)];
            nlev[size_t(j)] += hs[size_t(k)]->levels[size_t(l)].op.A.n;
        }
    for (int64_t n : nlev)
        if (n >= (int64_t(1) << 31) - kItemRows) throw Error(5, "batch level too large for 32-bit rows");
    // fine space (problem order)
    F_.assign(size_t(K) + 1, 0);
    for (int k = 0; k < K; ++k) F_[size_t(k) + 1] = F_[size_t(k)] + hs[size_t(k)]->levels[0].op.A.n;
    if (F_[size_t(K)] >= (int64_t(1) << 31) - kItemRows) throw Error(5, "batch too large for 32-bit rows");
    nfine_ = F_[size_t(K)];

    lev_.clear();
    lev_.resize(size_t(Lmax));
    int64_t max_items = 0;
    for (int j = 0; j < Lmax; ++j) {
        BLevelHost& H = lev_[size_t(j)];
        H.n = int(nlev[size_t(j)]);
        std::vector<int> rp(1, 0), ci, cptr, child;
        std::vector<double> val, wd, td, vol, cvol(size_t(K), 0.0);
        std::vector<BItem> items;
        std::vector<int> pfirst(size_t(K), 0), pcount(size_t(K), 0);
        for (int k = 0; k < K; ++k) {
            const Hierarchy& h = *hs[size_t(k)];
            const int Lk = int(h.levels.size());
            const int l = j - (Lmax - Lk);
            if (l < 0) continue;
            const HostLevel& hl = h.levels[size_t(l)];
            const Csr& A = hl.op.A;
            const int off = int(M[size_t(j)][size_t(k)]);
            for (int64_t i = 0; i < A.n; ++i) {
                for (int64_t q = A.ptr[size_t(i)]; q < A.ptr[size_t(i) + 1]; ++q) {
                    ci.push_back(A.col[size_t(q)] + off);
                    val.push_back(A.val[size_t(q)]);
                }
                rp.push_back(int(ci.size()));
                wd.push_back(hl.weight * hl.inv_diag[size_t(i)]);
                td.push_back(hl.transfer_inv.empty() ? 0.0 : hl.transfer_weight * hl.transfer_inv[size_t(i)]);
                vol.push_back(hl.op.volumes[size_t(i)]);
            }
            if (ci.size() >= size_t(1) << 31) throw Error(5, "batch level has too many nonzeros");
            if (hl.op.singular && !hl.op.comp.volume.empty()) cvol[size_t(k)] = 1.0 / hl.op.comp.volume[0];
            pfirst[size_t(k)] = int(items.size());
            const int delta = l == 0 ? int(F_[size_t(k)] - off) : kNoExt;
            for (int64_t b = 0; b < A.n; b += kItemRows)
                items.push_back(BItem{off + int(b), off + int(std::min<int64_t>(A.n, b + kItemRows)), k, delta});
            pcount[size_t(k)] = int(items.size()) - pfirst[size_t(k)];
        }
        H.nitems = int(items.size());
        max_items = std::max<int64_t>(max_items, H.nitems);
        // children of the next level's rows
        if (j + 1 < Lmax) {
            const int nc = int(nlev[size_t(j) + 1]);
            cptr.assign(size_t(nc) + 1, 0);
            // rows of problems absent from level j+1 have no owner; problems present
            // on level j are present on j+1 unless level j is their coarsest
            std::vector<int> own_full(size_t(H.n), -1);
            {
                for (int k = 0; k < K; ++k) {
                    const Hierarchy& h = *hs[size_t(k)];
                    const int Lk = int(h.levels.size());
                    const int l = j - (Lmax - Lk);
                    if (l < 0) continue;
                    const int off = int(M[size_t(j)][size_t(k)]);
                    const HostLevel& hl = h.levels[size_t(l)];
                    if (l + 1 < Lk) {
                        const int coff = int(M[size_t(j) + 1][size_t(k)]);
                        for (size_t i = 0; i < hl.owner.size(); ++i) own_full[size_t(off) + i] = hl.owner[i] + coff;
                    }
                }
            }
            for (int o : own_full)
                if (o >= 0) cptr[size_t(o) + 1]++;
            for (int c = 0; c < nc; ++c) cptr[size_t(c) + 1] += cptr[size_t(c)];
            child.assign(size_t(cptr[size_t(nc)]), 0);
            std::vector<int> nxt(cptr.begin(), cptr.end() - 1);
            for (int i = 0; i < H.n; ++i)
                if (own_full[size_t(i)] >= 0) child[size_t(nxt[size_t(own_full[size_t(i)])]++)] = i;
            H.owner.upload(own_full.data(), own_full.size(), stream_);
            H.cptr.upload(cptr.data(), cptr.size(), stream_);
            H.child.upload(child.data(), child.size(), stream_);
        }
        H.rp.upload(rp.data(), rp.size(), stream_);
        H.ci.upload(ci.data(), ci.size(), stream_);
        H.items.upload(items.data(), items.size(), stream_);
        H.pfirst.upload(pfirst.data(), pfirst.size(), stream_);
        H.pcount.upload(pcount.data(), pcount.size(), stream_);
        H.cvol_inv.upload(cvol.data(), cvol.size(), stream_);
        H.lsum.alloc(size_t(K));
        H.val_d.upload(val.data(), val.size(), stream_);
        H.wd_d.upload(wd.data(), wd.size(), stream_);
        H.td_d.upload(td.data(), td.size(), stream_);
        H.vol_d.upload(vol.data(), vol.size(), stream_);
        {
            auto f = cast_vec<float>(val);
            H.val_f.upload(f.data(), f.size(), stream_);
            auto g = cast_vec<float>(wd);
            H.wd_f.upload(g.data(), g.size(), stream_);
            auto t = cast_vec<float>(td);
            H.td_f.upload(t.data(), t.size(), stream_);
            auto v = cast_vec<float>(vol);
            H.vol_f.upload(v.data(), v.size(), stream_);
            TPA_CUDA(cudaStreamSynchronize(stream_));
        }
        for (auto* a : {&H.b_d, &H.bp_d, &H.x_d, &H.y_d, &H.r_d, &H.s_d}) a->alloc(size_t(H.n));
        for (auto* a : {&H.b_f, &H.bp_f, &H.x_f, &H.y_f, &H.r_f, &H.s_f}) a->alloc(size_t(H.n));
        TPA_CUDA(cudaStreamSynchronize(stream_));
    }
    // views
    vd_.assign(size_t(Lmax), BLevel<double>{});
    vf_.assign(size_t(Lmax), BLevel<float>{});
    for (int j = 0; j < Lmax; ++j) {
        BLevelHost& H = lev_[size_t(j)];
        auto fill = [&](auto& v, auto& val, auto& wd, auto& td, auto& vol, auto& b, auto& bp, auto& x, auto& y,
                        auto& r, auto& s) {
            v.n = H.n;
            v.nitems = H.nitems;
            v.items = H.items.p;
            v.rp = H.rp.p;
            v.ci = H.ci.p;
            v.val = val.p;
            v.wd = wd.p;
            v.td = td.p;
            v.vol = vol.p;
            v.owner = H.owner.p;
            v.cptr = H.cptr.p;
            v.child = H.child.p;
            v.cvol_inv = H.cvol_inv.p;
            v.pfirst = H.pfirst.p;
            v.pcount = H.pcount.p;
            v.lsum = H.lsum.p;
            v.b = b.p;
            v.bp = bp.p;
            v.x = x.p;
            v.y = y.p;
            v.r = r.p;
            v.s = s.p;
        };
        fill(vd_[size_t(j)], H.val_d, H.wd_d, H.td_d, H.vol_d, H.b_d, H.bp_d, H.x_d, H.y_d, H.r_d, H.s_d);
        fill(vf_[size_t(j)], H.val_f, H.wd_f, H.td_f, H.vol_f, H.b_f, H.bp_f, H.x_f, H.y_f, H.r_f, H.s_f);
    }
    vd_dev_.upload(vd_.data(), vd_.size(), stream_);
    vf_dev_.upload(vf_.data(), vf_.size(), stream_);
    // tails and coarse inverses
    {
        std::vector<double> G;
        std::vector<int64_t> goff(static_cast<size_t>(K));
        for (int k = 0; k < K; ++k) {
            goff[size_t(k)] = int64_t(G.size());
            G.insert(G.end(), hs[size_t(k)]->coarse_inverse.begin(), hs[size_t(k)]->coarse_inverse.end());
        }
        G_.upload(G.data(), G.size(), stream_);
        TPA_CUDA(cudaStreamSynchronize(stream_));
        std::vector<BTail> tails(static_cast<size_t>(K));
        for (int k = 0; k < K; ++k) {
            BTail& t = tails[size_t(k)];
            std::memset(&t, 0, sizeof(t));
            for (int q = 0; q < T; ++q) {
                const int j = Lmax - T + q;
                const int64_t off = M[size_t(j)][size_t(k)];
                const Hierarchy& h = *hs[size_t(k)];
                const int l = j - (Lmax - int(h.levels.size()));
                t.begin[q] = int(off);
                t.end[q] = int(off + h.levels[size_t(l)].op.A.n);
            }
            t.G = G_.p + goff[size_t(k)];
            t.gn = int(hs[size_t(k)]->coarse_n);
        }
        tails_.upload(tails.data(), tails.size(), stream_);
    }
    // fine space: items, FP64 CSR and volumes
    {
        std::vector<BFItem> fi;
        std::vector<int> pf(static_cast<size_t>(K)), pc(static_cast<size_t>(K)), rp(1, 0), ci;
        std::vector<double> val, vol;
        for (int k = 0; k < K; ++k) {
            const Hierarchy& h = *hs[size_t(k)];
            const int Lk = int(h.levels.size());
            const int j = Lmax - Lk;
            const Csr& A = h.levels[0].op.A;
            const int F = int(F_[size_t(k)]);
            const int off = int(M[size_t(j)][size_t(k)]) - F;
            pf[size_t(k)] = int(fi.size());
            for (int64_t b = 0; b < A.n; b += kItemRows)
                fi.push_back(BFItem{F + int(b), F + int(std::min<int64_t>(A.n, b + kItemRows)), k, j, off});
            pc[size_t(k)] = int(fi.size()) - pf[size_t(k)];
            for (int64_t i = 0; i < A.n; ++i) {
                for (int64_t q = A.ptr[size_t(i)]; q < A.ptr[size_t(i) + 1]; ++q) {
                    ci.push_back(A.col[size_t(q)] + F);
                    val.push_back(A.val[size_t(q)]);
                }
                rp.push_back(int(ci.size()));
            }
            vol.insert(vol.end(), h.levels[0].op.volumes.begin(), h.levels[0].op.volumes.end());
            comp_vol_.push_back(h.levels[0].op.singular ? h.levels[0].op.comp.volume[0] : 0.0);
            double tv = 0;
            for (double v : h.levels[0].op.volumes)
                if (v > 0) tv += v;
            total_vol_.push_back(tv);
        }
        nfi_ = int(fi.size());
        max_items = std::max<int64_t>(max_items, nfi_);
        fitems_.upload(fi.data(), fi.size(), stream_);
        fpfirst_.upload(pf.data(), pf.size(), stream_);
        fpcount_.upload(pc.data(), pc.size(), stream_);
        frp_.upload(rp.data(), rp.size(), stream_);
        fci_.upload(ci.data(), ci.size(), stream_);
        fval_.upload(val.data(), val.size(), stream_);
        fvol_.upload(vol.data(), vol.size(), stream_);
        TPA_CUDA(cudaStreamSynchronize(stream_));
    }
    const size_t nf = size_t(nfine_);
    for (auto* a : {&b_, &x_, &r_, &p_, &ap_, &z_, &rhs_, &x0_}) a->alloc(nf);
    partial_.alloc(size_t(max_items));
    partial2_.alloc(size_t(max_items));
    counters_.alloc(size_t(bcCount) * size_t(K));
    TPA_CUDA(cudaMemsetAsync(counters_.p, 0, counters_.n * sizeof(unsigned), stream_));
    state_.alloc(size_t(K));
    active_.alloc(size_t(K));
    mean_.alloc(size_t(K));
    kvec_.alloc(size_t(8) * size_t(K));
    kint_.alloc(size_t(K));
    TPA_CUDA(cudaMemsetAsync(mean_.p, 0, size_t(K) * sizeof(double), stream_));
    TPA_CUDA(cudaStreamSynchronize(stream_));
}

// ---- one V-cycle of every active problem ------------------------------------------

template <typename T>
void BatchSolver::enqueue_vcycle(const double* r) {
    const Launch go{stream_, true};
    const std::vector<BLevel<T>>* Vp;
    const BLevel<T>* Vdev;
    if constexpr (std::is_same<T, double>::value) {
        Vp = &vd_;
        Vdev = vd_dev_.p;
    } else {
        Vp = &vf_;
        Vdev = vf_dev_.p;
    }
    const std::vector<BLevel<T>>& V = *Vp;
    const int top = L_ - T_;  // first tail level
    BState* st = state_.p;
    unsigned* cr = counters_.p + size_t(bcRestrict) * size_t(K_);
    unsigned* cp = counters_.p + size_t(bcPost) * size_t(K_);
    for (int j = 0; j < top; ++j) {
        const BLevel<T>& L = V[size_t(j)];
        go(bk_pre2<T>, L.nitems, kItemRows, 0, L, r, st, active_.p);
        go(bk_residual<T>, L.nitems, kItemRows, 0, L, active_.p);
        go(bk_restrict<T>, V[size_t(j) + 1].nitems, kItemRows, 0, L, V[size_t(j) + 1], partial_.p, cr, active_.p);
        launches_ += 3;
    }
    go(bk_tail<T>, K_, kTailThreads, 0, Vdev, top, T_, tails_.p, active_.p);
    ++launches_;
    for (int j = top - 1; j >= 0; --j) {
        const BLevel<T>& L = V[size_t(j)];
        go(bk_prolong<T>, L.nitems, kItemRows, 0, L, V[size_t(j) + 1].x, active_.p);
        go(bk_post1<T>, L.nitems, kItemRows, 0, L, active_.p);
        go(bk_post2<T>, L.nitems, kItemRows, 0, L, partial_.p, cp, mean_.p, active_.p);
        launches_ += 3;
    }
}

void BatchSolver::enqueue_z(int precision, int init) {
    const Launch go{stream_, true};
    BState* st = state_.p;
    unsigned* cz = counters_.p + size_t(bcZ) * size_t(K_);
    if (precision == 0)
        go(bk_cg_z<double>, nfi_, kItemRows, 0, fitems_.p, fpfirst_.p, fpcount_.p, vd_dev_.p, mean_.p, r_.p, z_.p,
           p_.p, partial_.p, cz, st, active_.p, init);
    else
        go(bk_cg_z<float>, nfi_, kItemRows, 0, fitems_.p, fpfirst_.p, fpcount_.p, vf_dev_.p, mean_.p, r_.p, z_.p,
           p_.p, partial_.p, cz, st, active_.p, init);
    ++launches_;
}

void BatchSolver::enqueue_body(int precision, cudaGraphConditionalHandle handle, bool in_graph) {
    const Launch go{stream_, true};
    BState* st = state_.p;
    const FineCsr A{frp_.p, fci_.p, fval_.p, fvol_.p};
    go(bk_cg_ap, nfi_, kItemRows, 0, fitems_.p, fpfirst_.p, fpcount_.p, A, p_.p, ap_.p, partial_.p,
       counters_.p + size_t(bcAp) * size_t(K_), st, active_.p);
    go(bk_cg_update, nfi_, kItemRows, 0, fitems_.p, fpfirst_.p, fpcount_.p, fvol_.p, x_.p, r_.p, p_.p, ap_.p,
       partial_.p, partial2_.p, counters_.p + size_t(bcUpdMax) * size_t(K_),
       counters_.p + size_t(bcUpdSum) * size_t(K_), st, active_.p);
    launches_ += 2;
    if (precision == 0) enqueue_vcycle<double>(r_.p);
    else enqueue_vcycle<float>(r_.p);
    enqueue_z(precision, 0);
    go(bk_cg_p, nfi_, kItemRows, 0, fitems_.p, p_.p, z_.p, st, active_.p);
    ++launches_;
    if (in_graph) {
        go(bk_cg_cond, 1, 256, 0, active_.p, K_, handle);
        ++launches_;
    }
}

cudaGraphExec_t BatchSolver::graph(int precision) {
    if (exec_[precision]) return exec_[precision];
    cudaGraph_t g;
    TPA_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle handle;
    TPA_CUDA(cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault));
    alignas(cudaGraphNodeParams) unsigned char storage[sizeof(cudaGraphNodeParams)];
    std::memset(storage, 0, sizeof(storage));
    cudaGraphNodeParams& cp = *reinterpret_cast<cudaGraphNodeParams*>(storage);
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    TPA_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    cudaStream_t saved = stream_;
    stream_ = own_stream_;
    const int before = launches_;
    TPA_CUDA(cudaStreamBeginCaptureToGraph(stream_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    enqueue_body(precision, handle, true);
    cudaGraph_t captured;
    cudaError_t ce = cudaStreamEndCapture(stream_, &captured);
    stream_ = saved;
    body_launches_[precision] = launches_ - before;
    launches_ = before;
    if (ce != cudaSuccess) {
        cudaGraphDestroy(g);
        throw Error(2, std::string("batch graph capture failed: ") + cudaGetErrorString(ce));
    }
    cudaGraphExec_t exec;
    cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) throw Error(2, std::string("batch graph instantiation failed: ") + cudaGetErrorString(ie));
    exec_[precision] = exec;
    return exec;
}

// ---- the solve --------------------------------------------------------------------

void BatchSolver::solve(const double* rhs, double* x_user, double rtol, double atol, int max_cycles,
                        int compatibility, int precision, std::vector<SolveStats>& stats, std::vector<int>& status,
                        std::vector<std::string>& messages) {
    TPA_CUDA(cudaSetDevice(device_));
    if (!(rtol >= 0 && rtol < 1)) throw Error(1, "rtol must lie in [0, 1)");
    if (!(atol >= 0)) throw Error(1, "atol must be nonnegative");
    if (max_cycles < 0) throw Error(1, "max_cycles must be nonnegative");
    if (compatibility != 0 && compatibility != 1) throw Error(1, "compatibility must be :project or :error");
    if (precision != 0 && precision != 1) throw Error(1, "precision must be 0 (FP64) or 1 (mixed)");
    const double eps = 2.220446049250313e-16;
    const int K = K_;
    const Launch go{stream_, false};
    const FineCsr A{frp_.p, fci_.p, fval_.p, fvol_.p};
    BState* st = state_.p;
    stats.assign(size_t(K), SolveStats());
    status.assign(size_t(K), 0);
    messages.assign(size_t(K), std::string());
    cudaEvent_t e0, e1;
    TPA_CUDA(cudaEventCreate(&e0));
    TPA_CUDA(cudaEventCreate(&e1));
    TPA_CUDA(cudaEventRecord(e0, stream_));
    std::vector<double> h(size_t(8) * size_t(K));
    double* d_a = kvec_.p;                // per-problem scratch vectors on the device
    double* d_b = kvec_.p + K;
    double* d_c = kvec_.p + 2 * K;
    double* d_coef = kvec_.p + 3 * K;
    double* d_target = kvec_.p + 4 * K;
    auto read = [&](const double* d, std::vector<double>& out) {
        out.resize(size_t(K));
        TPA_CUDA(cudaMemcpyAsync(out.data(), d, size_t(K) * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        TPA_CUDA(cudaStreamSynchronize(stream_));
    };
    auto write = [&](double* d, const std::vector<double>& in) {
        TPA_CUDA(cudaMemcpyAsync(d, in.data(), size_t(K) * sizeof(double), cudaMemcpyHostToDevice, stream_));
    };
    auto set_active = [&](const std::vector<int>& a) {
        TPA_CUDA(cudaMemcpyAsync(active_.p, a.data(), size_t(K) * sizeof(int), cudaMemcpyHostToDevice, stream_));
        TPA_CUDA(cudaStreamSynchronize(stream_));
    };
    unsigned* cs = counters_.p + size_t(bcSum) * size_t(K);
    unsigned* cm = counters_.p + size_t(bcMax) * size_t(K);
    auto sums = [&](const double* v, const double* w, int absval, double* out) {
        go(bk_sum, nfi_, kItemRows, 0, fitems_.p, fpfirst_.p, fpcount_.p, v, w, absval, partial_.p, cs, out);
        ++launches_;
    };
    // x mean removal for the problems with sel[k]
    auto remove_means = [&](const std::vector<int>& sel) {
        sums(x_.p, fvol_.p, 0, d_a);
        std::vector<double> s;
        read(d_a, s);
        std::vector<double> coef(size_t(K), 0.0);
        for (int k = 0; k < K; ++k)
            if (sel[size_t(k)] && comp_vol_[size_t(k)] > 0) coef[size_t(k)] = s[size_t(k)] / comp_vol_[size_t(k)];
        write(d_coef, coef);
        go(bk_sub, nfi_, kItemRows, 0, fitems_.p, x_.p, (const double*)nullptr, d_coef);
        ++launches_;
    };
    auto residual_norms = [&](std::vector<double>& linf, std::vector<double>* l2) {
        go(bk_residual64, nfi_, kItemRows, 0, fitems_.p, fpfirst_.p, fpcount_.p, A, b_.p, x_.p, r_.p, partial2_.p,
           partial_.p, cm, cs, d_a, l2 ? d_b : (double*)nullptr, (BState*)nullptr, (const int*)nullptr);
        ++launches_;
        read(d_a, linf);
        if (l2) {
            std::vector<double> num;
            read(d_b, num);
            l2->resize(size_t(K));
            for (int k = 0; k < K; ++k) {
                const double tv = total_volume(k);
                (*l2)[size_t(k)] = tv > 0 ? std::sqrt(num[size_t(k)] / tv) : 0.0;
            }
        }
    };
    auto floors = [&](std::vector<double>& fl) {
        go(bk_abs_bound, nfi_, kItemRows, 0, fitems_.p, fpfirst_.p, fpcount_.p, A, b_.p, x_.p, partial2_.p, cm,
           d_c);
        ++launches_;
        read(d_c, fl);
        for (double& f : fl) f = 128 * eps * std::max(1.0, f);
    };

    // prepare: b = V f, x = x0, component projection, gauge of x
    TPA_CUDA(cudaMemcpyAsync(rhs_.p, rhs, size_t(nfine_) * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    TPA_CUDA(cudaMemcpyAsync(x0_.p, x_user, size_t(nfine_) * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    go(bk_prepare, nfi_, kItemRows, 0, fitems_.p, A, rhs_.p, x0_.p, b_.p, x_.p);
    ++launches_;
    std::vector<int> ok(size_t(K), 1), all(size_t(K), 1);
    {
        std::vector<double> s, sa;
        sums(b_.p, nullptr, 0, d_a);
        read(d_a, s);
        if (compatibility == 1) {
            sums(b_.p, nullptr, 1, d_b);
            read(d_b, sa);
        }
        std::vector<double> coef(size_t(K), 0.0);
        for (int k = 0; k < K; ++k) {
            if (comp_vol_[size_t(k)] <= 0) continue;
            if (compatibility == 1 && std::fabs(s[size_t(k)]) > 256 * eps * std::max(1.0, sa[size_t(k)])) {
                ok[size_t(k)] = 0;
                status[size_t(k)] = 1;
                messages[size_t(k)] = "Poisson right-hand side has nonzero volume mean";
                continue;
            }
            coef[size_t(k)] = s[size_t(k)] / comp_vol_[size_t(k)];
            stats[size_t(k)].removed_rhs_mean = coef[size_t(k)];
            stats[size_t(k)].removed_max_component_mean = std::fabs(coef[size_t(k)]);
        }
        write(d_coef, coef);
        go(bk_sub, nfi_, kItemRows, 0, fitems_.p, b_.p, fvol_.p, d_coef);
        ++launches_;
        remove_means(all);
    }
    std::vector<double> init_linf, init_l2, floor;
    residual_norms(init_linf, &init_l2);
    floors(floor);
    std::vector<double> target(static_cast<size_t>(K));
    std::vector<int> total(size_t(K), 0), run(size_t(K), 0);
    for (int k = 0; k < K; ++k) {
        target[size_t(k)] = std::max(atol, std::max(rtol * std::max(init_linf[size_t(k)], eps), floor[size_t(k)]));
        run[size_t(k)] = ok[size_t(k)] && init_linf[size_t(k)] > target[size_t(k)] && max_cycles > 0;
    }
    auto guarded = [&](int k, const std::vector<double>& fl, double cur) {
        const double init = init_linf[size_t(k)], tg = target[size_t(k)];
        if (!(std::isfinite(init) && std::isfinite(cur) && tg < cur && cur < init)) return tg;
        const double f = fl[size_t(k)];
        return (std::isfinite(f) && f < init / 100) ? std::max(tg, f) : tg;
    };
    while (std::any_of(run.begin(), run.end(), [](int v) { return v != 0; })) {
        // one Krylov run of every problem in `run`
        std::vector<double> itmax_d(static_cast<size_t>(K));
        std::vector<int> itmax(static_cast<size_t>(K));
        for (int k = 0; k < K; ++k) itmax[size_t(k)] = max_cycles - total[size_t(k)];
        TPA_CUDA(cudaMemcpyAsync(kint_.p, itmax.data(), size_t(K) * sizeof(int), cudaMemcpyHostToDevice, stream_));
        write(d_target, target);
        go(bk_state_init, (K + 255) / 256, 256, 0, st, d_target, kint_.p, K);
        set_active(run);
        const Launch gp{stream_, true};
        gp(bk_residual64, nfi_, kItemRows, 0, fitems_.p, fpfirst_.p, fpcount_.p, A, b_.p, x_.p, r_.p, partial2_.p,
           partial_.p, cm, cs, (double*)nullptr, (double*)nullptr, st, active_.p);
        launches_ += 2;
        if (precision == 0) enqueue_vcycle<double>(r_.p);
        else enqueue_vcycle<float>(r_.p);
        enqueue_z(precision, 1);
        std::vector<int> act(static_cast<size_t>(K));
        TPA_CUDA(cudaMemcpyAsync(act.data(), active_.p, size_t(K) * sizeof(int), cudaMemcpyDeviceToHost, stream_));
        TPA_CUDA(cudaStreamSynchronize(stream_));
        const bool no_graph = std::getenv("TPAGMG_NO_GRAPH") != nullptr;
        if (std::any_of(act.begin(), act.end(), [](int v) { return v != 0; })) {
            if (no_graph) {
                // the same body launched kernel by kernel, the loop condition
                // read on the host after each body (profiling and diagnosis);
                // every problem stops within its iteration limit
                for (int body = 0; body <= max_cycles; ++body) {
                    enqueue_body(precision, cudaGraphConditionalHandle(), false);
                    TPA_CUDA(cudaMemcpyAsync(act.data(), active_.p, size_t(K) * sizeof(int), cudaMemcpyDeviceToHost,
                                             stream_));
                    TPA_CUDA(cudaStreamSynchronize(stream_));
                    if (std::none_of(act.begin(), act.end(), [](int v) { return v != 0; })) break;
                }
            } else {
                cudaGraphExec_t exec = graph(precision);
                TPA_CUDA(cudaGraphLaunch(exec, stream_));
            }
        }
        std::vector<BState> hs(static_cast<size_t>(K));
        TPA_CUDA(cudaMemcpyAsync(hs.data(), st, size_t(K) * sizeof(BState), cudaMemcpyDeviceToHost, stream_));
        TPA_CUDA(cudaStreamSynchronize(stream_));
        int max_iter = 0;
        for (int k = 0; k < K; ++k)
            if (run[size_t(k)]) max_iter = std::max(max_iter, hs[size_t(k)].iter + ((hs[size_t(k)].flags & 2) ? 1 : 0));
        if (!no_graph) launches_ += max_iter * body_launches_[precision];
        remove_means(run);
        std::vector<double> fin, fl;
        residual_norms(fin, nullptr);
        floors(fl);
        for (int k = 0; k < K; ++k) {
            if (!run[size_t(k)]) continue;
            const int niter = hs[size_t(k)].iter;
            total[size_t(k)] += niter;
            stats[size_t(k)].restarts += 1;
            const double eff = guarded(k, fl, fin[size_t(k)]);
            const bool done = fin[size_t(k)] <= eff || !std::isfinite(fin[size_t(k)]) || niter == 0 ||
                              total[size_t(k)] >= max_cycles;
            if (done) run[size_t(k)] = 0;
        }
    }
    remove_means(ok);
    std::vector<double> fin_linf, fin_l2, fl;
    residual_norms(fin_linf, &fin_l2);
    floors(fl);
    go(bk_copy_out, nfi_, kItemRows, 0, fitems_.p, x_.p, x_user);
    ++launches_;
    TPA_CUDA(cudaEventRecord(e1, stream_));
    TPA_CUDA(cudaEventSynchronize(e1));
    TPA_CUDA(cudaGetLastError());
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (int k = 0; k < K; ++k) {
        SolveStats& s = stats[size_t(k)];
        const double tg = guarded(k, fl, fin_linf[size_t(k)]);
        s.cycles = total[size_t(k)];
        s.converged = ok[size_t(k)] && std::isfinite(fin_linf[size_t(k)]) && std::isfinite(tg) &&
                      fin_linf[size_t(k)] <= tg;
        s.initial_l2 = init_l2[size_t(k)];
        s.initial_linf = init_linf[size_t(k)];
        s.final_l2 = fin_l2[size_t(k)];
        s.final_linf = fin_linf[size_t(k)];
        s.target_linf = tg;
        s.residual_scale = std::max(init_linf[size_t(k)], eps);
        s.ms_total = ms;
    }
    last_ms_ = ms;
}

double BatchSolver::total_volume(int k) const {
    return total_vol_.empty() ? 0.0 : total_vol_[size_t(k)];
}

template void BatchSolver::enqueue_vcycle<double>(const double*);
template void BatchSolver::enqueue_vcycle<float>(const double*);

}  // namespace tpa
