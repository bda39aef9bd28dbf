// Vectorized kernels for constant-coefficient levels of 16x16 blocks (uniform
// regions of the tree, e.g. every level of a periodic uniform mesh).
//
// A CTA of 256 threads covers 4 blocks; a thread owns a 4-cell row segment
// ("quad") of one block: row j = (t % 64) / 4, cells 4q .. 4q+3 with q = t % 4.
// Its own, southern and northern quads are 16-byte (FP32) or 2 x 16-byte
// (FP64) loads; the western / eastern neighbour values come from the adjacent
// lanes by warp shuffles, and across a block edge from the neighbour block
// (W/E/S/N table, -1: wall).  Every stencil coefficient equals c0, so a
// matrix row is c0 * (count * v_c - sum of neighbours).
//
// The phases are those of stencil.cuh (the default V-cycle of
// src/solvers/multigrid/cycles.jl:46-77, ronaldremmerswaal/TwoPhaseAMR.jl), with
// the same deferred mean handling; only the data movement differs.
#pragma once

#include <cuda_runtime.h>

#include "stencil.cuh"

namespace tpa {

template <typename T>
struct Quad {
    T v[4];
};

__device__ __forceinline__ Quad<float> q_ld(const float* p) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    return Quad<float>{{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ Quad<double> q_ld(const double* p) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return Quad<double>{{a.x, a.y, b.x, b.y}};
}
// loads of data written by an earlier kernel of the same cycle (no read-only path)
__device__ __forceinline__ Quad<float> q_ldv(const float* p) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    return Quad<float>{{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ Quad<double> q_ldv(const double* p) {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    return Quad<double>{{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void q_st(float* p, const Quad<float>& q) {
    *reinterpret_cast<float4*>(p) = make_float4(q.v[0], q.v[1], q.v[2], q.v[3]);
}
__device__ __forceinline__ void q_st(double* p, const Quad<double>& q) {
    reinterpret_cast<double2*>(p)[0] = make_double2(q.v[0], q.v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(q.v[2], q.v[3]);
}
// FP64 values stored as FP32 (round to nearest)
__device__ __forceinline__ void q_st(float* p, const Quad<double>& q) {
    *reinterpret_cast<float4*>(p) = make_float4(float(q.v[0]), float(q.v[1]), float(q.v[2]), float(q.v[3]));
}

// Position of a thread's quad.
struct QPos {
    int b, j, q, c;  // block, row, quad index, first cell
};

__device__ __forceinline__ QPos q_pos(int group) {
    const int t = threadIdx.x;
    QPos p;
    p.b = group * 4 + (t >> 6);
    p.j = (t & 63) >> 2;
    p.q = t & 3;
    p.c = p.b * 256 + p.j * 16 + 4 * p.q;
    return p;
}

// A quad and its neighbours for the stencil (missing neighbours: flag false).
template <typename T>
struct QNb {
    Quad<T> x, s, n;
    T w, e;
    bool hs, hn, hw, he;
};

// Load the stencil neighbourhood of a quad of `v`, with `f` applied to every
// loaded value (f(value, cell)).  All lanes of the warp must call it (shuffles);
// lanes of blocks beyond the level pass valid = false and get zeros.
template <typename T, typename Ld, typename F>
__device__ __forceinline__ QNb<T> q_gather(const SView<T>& L, const QPos& p, bool valid, Ld ld, F f) {
    QNb<T> r;
    r.hs = r.hn = r.hw = r.he = false;
    r.w = r.e = T(0);
    for (int m = 0; m < 4; ++m) r.x.v[m] = r.s.v[m] = r.n.v[m] = T(0);
    int nbW = -1, nbE = -1, nbS = -1, nbN = -1;
    if (valid) {
        const int4 nb = *reinterpret_cast<const int4*>(L.nbr + 4 * p.b);
        nbW = nb.x;
        nbE = nb.y;
        nbS = nb.z;
        nbN = nb.w;
        r.x = ld(p.c);
        for (int m = 0; m < 4; ++m) r.x.v[m] = f(r.x.v[m], p.c + m);
        int sc = -1, nc = -1;
        if (p.j > 0) sc = p.c - 16;
        else if (nbS >= 0) sc = nbS * 256 + 240 + 4 * p.q;
        if (p.j < 15) nc = p.c + 16;
        else if (nbN >= 0) nc = nbN * 256 + 4 * p.q;
        if (sc >= 0) {
            r.s = ld(sc);
            for (int m = 0; m < 4; ++m) r.s.v[m] = f(r.s.v[m], sc + m);
            r.hs = true;
        }
        if (nc >= 0) {
            r.n = ld(nc);
            for (int m = 0; m < 4; ++m) r.n.v[m] = f(r.n.v[m], nc + m);
            r.hn = true;
        }
    }
    // horizontal neighbours of the quad's end cells: the adjacent lanes' values
    const T left = __shfl_up_sync(0xffffffffu, r.x.v[3], 1);
    const T right = __shfl_down_sync(0xffffffffu, r.x.v[0], 1);
    if (valid) {
        if (p.q > 0) {
            r.w = left;
            r.hw = true;
        } else if (nbW >= 0) {
            const int wc = nbW * 256 + p.j * 16 + 15;
            r.w = f(ld(wc - 3).v[3], wc);
            r.hw = true;
        }
        if (p.q < 3) {
            r.e = right;
            r.he = true;
        } else if (nbE >= 0) {
            const int ec = nbE * 256 + p.j * 16;
            r.e = f(ld(ec).v[0], ec);
            r.he = true;
        }
    }
    return r;
}

// (A v) for the 4 cells of the quad
template <typename T>
__device__ __forceinline__ Quad<T> q_apply(const SView<T>& L, const QNb<T>& g) {
    Quad<T> out;
    for (int m = 0; m < 4; ++m) {
        const bool hw = m > 0 || g.hw, he = m < 3 || g.he;
        const T wv = m > 0 ? g.x.v[m - 1] : g.w;
        const T ev = m < 3 ? g.x.v[m + 1] : g.e;
        T off = T(0);
        int cnt = 0;
        if (hw) off += wv, ++cnt;
        if (he) off += ev, ++cnt;
        if (g.hs) off += g.s.v[m], ++cnt;
        if (g.hn) off += g.n.v[m], ++cnt;
        out.v[m] = L.c0 * (T(cnt) * g.x.v[m] - off);
    }
    return out;
}

template <typename T>
__device__ __forceinline__ Quad<T> q_dinv(const SView<T>& L, int c) {
    if (!L.dinv) return Quad<T>{{L.dinv0, L.dinv0, L.dinv0, L.dinv0}};
    return q_ld(L.dinv + c);
}

#define TPA_Q_LOOP(groups)                                                            \
    for (int grp = blockIdx.x; grp < (groups); grp += gridDim.x)

// both pre-sweeps from x = 0, with the level's RHS projection
template <typename T, typename TB>
__global__ void __launch_bounds__(256) v_pre2(SView<T> L, const TB* __restrict__ bin, const double* level_sum) {
    pdl_entry();
    const double mean = (L.singular && level_sum) ? *level_sum * L.cvol_inv : 0.0;
    const int groups = (L.nblocks + 3) / 4;
    TPA_Q_LOOP(groups) {
        const QPos p = q_pos(grp);
        const bool valid = p.b < L.nblocks;
        auto ldb = [&](int c) {
            Quad<T> r;
            const Quad<TB> a = q_ldv(bin + c);
            for (int m = 0; m < 4; ++m) r.v[m] = T(a.v[m]);
            if (mean != 0.0) {
                const Quad<T> v = L.const_vol ? Quad<T>{{L.vol0, L.vol0, L.vol0, L.vol0}} : q_ld(L.vol + c);
                for (int m = 0; m < 4; ++m) r.v[m] = T(double(a.v[m]) - double(v.v[m]) * mean);
            }
            return r;
        };
        // first sweep is pointwise: x1 = w D^-1 pb; the neighbours of the second need x1
        const QNb<T> gb = q_gather<T>(L, p, valid, ldb, [](T v, int) { return v; });
        QNb<T> gx = gb;
        auto scale = [&](T v, int c) { return L.w * (L.dinv ? L.dinv[c] : L.dinv0) * v; };
        for (int m = 0; m < 4; ++m) {
            gx.x.v[m] = valid ? scale(gb.x.v[m], p.c + m) : T(0);
            if (valid && gb.hs) gx.s.v[m] = scale(gb.s.v[m], (p.j > 0 ? p.c - 16 : 0) + m);
            if (valid && gb.hn) gx.n.v[m] = scale(gb.n.v[m], (p.j < 15 ? p.c + 16 : 0) + m);
        }
        if (L.dinv && valid) {
            // exact neighbour cells for a varying D^-1
            const int4 nb = *reinterpret_cast<const int4*>(L.nbr + 4 * p.b);
            if (gb.hs) {
                const int sc = p.j > 0 ? p.c - 16 : nb.z * 256 + 240 + 4 * p.q;
                for (int m = 0; m < 4; ++m) gx.s.v[m] = scale(gb.s.v[m], sc + m);
            }
            if (gb.hn) {
                const int nc = p.j < 15 ? p.c + 16 : nb.w * 256 + 4 * p.q;
                for (int m = 0; m < 4; ++m) gx.n.v[m] = scale(gb.n.v[m], nc + m);
            }
        }
        const T lw = __shfl_up_sync(0xffffffffu, gx.x.v[3], 1);
        const T re = __shfl_down_sync(0xffffffffu, gx.x.v[0], 1);
        if (valid) {
            const int4 nb = *reinterpret_cast<const int4*>(L.nbr + 4 * p.b);
            gx.w = p.q > 0 ? lw : (gb.hw ? scale(gb.w, nb.x * 256 + p.j * 16 + 15) : T(0));
            gx.e = p.q < 3 ? re : (gb.he ? scale(gb.e, nb.y * 256 + p.j * 16) : T(0));
            const Quad<T> ax = q_apply(L, gx);
            const Quad<T> d = q_dinv(L, p.c);
            Quad<T> x2;
            for (int m = 0; m < 4; ++m) x2.v[m] = gx.x.v[m] + L.w * d.v[m] * (gb.x.v[m] - ax.v[m]);
            q_st(L.x + p.c, x2);
            q_st(L.bp + p.c, gb.x);
        }
    }
}

// r = bp - A x, s = D^-1 r
template <typename T>
__global__ void __launch_bounds__(256) v_residual(SView<T> L) {
    pdl_entry();
    const int groups = (L.nblocks + 3) / 4;
    TPA_Q_LOOP(groups) {
        const QPos p = q_pos(grp);
        const bool valid = p.b < L.nblocks;
        const QNb<T> g = q_gather<T>(L, p, valid, [&](int c) { return q_ldv(L.x + c); }, [](T v, int) { return v; });
        if (!valid) continue;
        const Quad<T> ax = q_apply(L, g);
        const Quad<T> bp = q_ldv(L.bp + p.c);
        const Quad<T> d = q_dinv(L, p.c);
        Quad<T> r, s;
        for (int m = 0; m < 4; ++m) {
            r.v[m] = bp.v[m] - ax.v[m];
            s.v[m] = d.v[m] * r.v[m];
        }
        q_st(L.r + p.c, r);
        q_st(L.s + p.c, s);
    }
}

// b_c = P_tent'(r - wt A s): 2x2 (scale 2) or 1x1 (scale 1) aggregation into the
// coarse block's quadrant; optional fold of the coarse RHS sum
template <typename T>
__global__ void __launch_bounds__(256) v_restrict(SView<T> L, T* __restrict__ bc, double* partial, unsigned* counter,
                                                  double* coarse_sum) {
    pdl_entry();
    const int groups = (L.nblocks + 3) / 4;
    double part = 0;
    TPA_Q_LOOP(groups) {
        const QPos p = q_pos(grp);
        const bool valid = p.b < L.nblocks;
        const QNb<T> g = q_gather<T>(L, p, valid, [&](int c) { return q_ldv(L.s + c); }, [](T v, int) { return v; });
        Quad<T> t;
        for (int m = 0; m < 4; ++m) t.v[m] = T(0);
        int4 mp = make_int4(0, 0, 0, 0);
        if (valid) {
            const Quad<T> as = q_apply(L, g);
            const Quad<T> r = q_ldv(L.r + p.c);
            for (int m = 0; m < 4; ++m) t.v[m] = r.v[m] - L.tw * as.v[m];
            mp = *reinterpret_cast<const int4*>(L.map + 4 * p.b);
        }
        // horizontal pairs, then the row below (lane + 4 holds row j + 1)
        const T h0 = t.v[0] + t.v[1], h1 = t.v[2] + t.v[3];
        const T d0 = __shfl_down_sync(0xffffffffu, h0, 4);
        const T d1 = __shfl_down_sync(0xffffffffu, h1, 4);
        if (!valid) continue;
        if (mp.w == 1) {
            T* dst = bc + mp.x * 256 + (mp.z + p.j) * 16 + mp.y + 4 * p.q;
            for (int m = 0; m < 4; ++m) {
                dst[m] = t.v[m];
                part += double(t.v[m]);
            }
        } else if ((p.j & 1) == 0) {
            const T c0 = h0 + d0, c1 = h1 + d1;
            T* dst = bc + mp.x * 256 + (mp.z + (p.j >> 1)) * 16 + mp.y + 2 * p.q;
            dst[0] = c0;
            dst[1] = c1;
            part += double(c0) + double(c1);
        }
    }
    if (coarse_sum) {
        if (publish_partial(part, partial, counter)) {
            const double s = fold_partials(partial, gridDim.x);
            if (threadIdx.x == 0) {
                *coarse_sum = s;
                *counter = 0;
            }
        }
    }
}

// e = P_tent x_c for the quad of block b, row j (map: coarse block, ox, oy, scale)
template <typename T>
__device__ __forceinline__ Quad<T> q_coarse(const SView<T>& L, const T* xc, int b, int j, int q) {
    const int4 mp = *reinterpret_cast<const int4*>(L.map + 4 * b);
    if (mp.w == 1) {
        const T* src = xc + mp.x * 256 + (mp.z + j) * 16 + mp.y + 4 * q;
        return Quad<T>{{src[0], src[1], src[2], src[3]}};
    }
    const T* src = xc + mp.x * 256 + (mp.z + (j >> 1)) * 16 + mp.y + 2 * q;
    const T e0 = src[0], e1 = src[1];
    return Quad<T>{{e0, e0, e1, e1}};
}

template <typename T>
__device__ __forceinline__ T q_coarse_cell(const SView<T>& L, const T* xc, int b, int i, int j) {
    const int4 mp = *reinterpret_cast<const int4*>(L.map + 4 * b);
    if (mp.w == 1) return xc[mp.x * 256 + (mp.z + j) * 16 + mp.y + i];
    return xc[mp.x * 256 + (mp.z + (j >> 1)) * 16 + mp.y + (i >> 1)];
}

// x += e - wt D^-1 A e, e = P_tent x_c
template <typename T>
__global__ void __launch_bounds__(256) v_prolong(SView<T> L, const T* __restrict__ xc) {
    pdl_entry();
    const int groups = (L.nblocks + 3) / 4;
    TPA_Q_LOOP(groups) {
        const QPos p = q_pos(grp);
        const bool valid = p.b < L.nblocks;
        QNb<T> g;
        g.hs = g.hn = g.hw = g.he = false;
        g.w = g.e = T(0);
        for (int m = 0; m < 4; ++m) g.x.v[m] = g.s.v[m] = g.n.v[m] = T(0);
        int4 nb = make_int4(-1, -1, -1, -1);
        if (valid) {
            nb = *reinterpret_cast<const int4*>(L.nbr + 4 * p.b);
            g.x = q_coarse(L, xc, p.b, p.j, p.q);
            if (p.j > 0) {
                g.s = q_coarse(L, xc, p.b, p.j - 1, p.q);
                g.hs = true;
            } else if (nb.z >= 0) {
                g.s = q_coarse(L, xc, nb.z, 15, p.q);
                g.hs = true;
            }
            if (p.j < 15) {
                g.n = q_coarse(L, xc, p.b, p.j + 1, p.q);
                g.hn = true;
            } else if (nb.w >= 0) {
                g.n = q_coarse(L, xc, nb.w, 0, p.q);
                g.hn = true;
            }
        }
        const T lw = __shfl_up_sync(0xffffffffu, g.x.v[3], 1);
        const T re = __shfl_down_sync(0xffffffffu, g.x.v[0], 1);
        if (!valid) continue;
        if (p.q > 0) {
            g.w = lw;
            g.hw = true;
        } else if (nb.x >= 0) {
            g.w = q_coarse_cell(L, xc, nb.x, 15, p.j);
            g.hw = true;
        }
        if (p.q < 3) {
            g.e = re;
            g.he = true;
        } else if (nb.y >= 0) {
            g.e = q_coarse_cell(L, xc, nb.y, 0, p.j);
            g.he = true;
        }
        const Quad<T> ae = q_apply(L, g);
        const Quad<T> d = q_dinv(L, p.c);
        Quad<T> x = q_ldv(L.x + p.c);
        for (int m = 0; m < 4; ++m) x.v[m] += g.x.v[m] - L.tw * d.v[m] * ae.v[m];
        q_st(L.x + p.c, x);
    }
}

// out = in + w D^-1 (bp - A in); with `partial`, folds the volume-weighted sum of
// out into mean_out (times cvol_inv)
template <typename T, bool Fold, typename Epi = MeanOnly>
__global__ void __launch_bounds__(256) v_sweep(SView<T> L, const T* __restrict__ in, T* __restrict__ out,
                                               double* partial, unsigned* counter, double* mean_out,
                                               Epi epi = Epi()) {
    pdl_entry();
    const int groups = (L.nblocks + 3) / 4;
    double part = 0, rx = 0;
    TPA_Q_LOOP(groups) {
        const QPos p = q_pos(grp);
        const bool valid = p.b < L.nblocks;
        const QNb<T> g = q_gather<T>(L, p, valid, [&](int c) { return q_ldv(in + c); }, [](T v, int) { return v; });
        if (!valid) continue;
        const Quad<T> ax = q_apply(L, g);
        const Quad<T> bp = q_ldv(L.bp + p.c);
        const Quad<T> d = q_dinv(L, p.c);
        Quad<T> o;
        for (int m = 0; m < 4; ++m) o.v[m] = g.x.v[m] + L.w * d.v[m] * (bp.v[m] - ax.v[m]);
        q_st(out + p.c, o);
        if (Fold && mean_out) {
            const Quad<T> v = L.const_vol ? Quad<T>{{L.vol0, L.vol0, L.vol0, L.vol0}} : q_ld(L.vol + p.c);
            for (int m = 0; m < 4; ++m) part += double(v.v[m]) * double(o.v[m]);
            if constexpr (Epi::kRz) {
                const Quad<double> rq = q_ldv(epi.r + p.c);
                for (int m = 0; m < 4; ++m) rx += rq.v[m] * double(o.v[m]);
            }
        }
    }
    if (Fold && mean_out) fold_mean(part, rx, partial, counter, mean_out, L.cvol_inv, epi);
}

// finest level, FP64: y = A x with x'y folded by `fold`
template <typename Fold>
__device__ __forceinline__ void v_apply_dot(const SView<double>& L, const double* x, double* y, double* partial,
                                            unsigned* counter, Fold fold) {
    const int groups = (L.nblocks + 3) / 4;
    double part = 0;
    TPA_Q_LOOP(groups) {
        const QPos p = q_pos(grp);
        const bool valid = p.b < L.nblocks;
        const QNb<double> g =
            q_gather<double>(L, p, valid, [&](int c) { return q_ldv(x + c); }, [](double v, int) { return v; });
        if (!valid) continue;
        const Quad<double> ax = q_apply(L, g);
        q_st(y + p.c, ax);
        for (int m = 0; m < 4; ++m) part += g.x.v[m] * ax.v[m];
    }
    if (publish_partial(part, partial, counter)) {
        const double s = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            fold(s);
            *counter = 0;
        }
    }
}

// v_apply_dot with the operand formed where it is read: ld(c) is the quad of
// the operand at cells c .. c+3, and the CTA's own quads are stored to `keep`
// (P: the storage type of the operand and the product; FP32 storage takes an
// operand that ld has already rounded to FP32, so the product is that of the
// stored operand)
template <typename P, typename Ld, typename Fold>
__device__ __forceinline__ void v_apply_dot_ld(const SView<double>& L, Ld ld, P* keep, P* y, double* partial,
                                               unsigned* counter, Fold fold) {
    const int groups = (L.nblocks + 3) / 4;
    double part = 0;
    TPA_Q_LOOP(groups) {
        const QPos p = q_pos(grp);
        const bool valid = p.b < L.nblocks;
        const QNb<double> g = q_gather<double>(L, p, valid, ld, [](double v, int) { return v; });
        if (!valid) continue;
        const Quad<double> ax = q_apply(L, g);
        q_st(keep + p.c, g.x);
        q_st(y + p.c, ax);
        for (int m = 0; m < 4; ++m) part += g.x.v[m] * ax.v[m];
    }
    if (publish_partial(part, partial, counter)) {
        const double s = fold_partials(partial, gridDim.x);
        if (threadIdx.x == 0) {
            fold(s);
            *counter = 0;
        }
    }
}

#undef TPA_Q_LOOP

}  // namespace tpa
