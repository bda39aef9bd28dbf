// Row-streaming halves of the V-cycle for periodic constant-coefficient 16x16
// levels (tpa_tune_config.tiles = 4 or 5).
//
// The level is a full rectangle of nbx x nby blocks in row-major order (the
// mesh's (level, j, i) sort of a single-level leaf set), periodic on both axes,
// with one stencil coefficient c0, one inverse diagonal dinv0 and one cell
// volume, and the next level is the same lattice halved.  A cell is then
// addressed by its lattice position alone.
//
// A warp owns a strip of kStreamCols interior columns with a four-cell frame on
// each side: lane l holds the column pair x0 - 4 + 2 l and the one after it (a
// pair never straddles a block, so it is one 8- or 16-byte access).  The strip
// has ROWS interior rows (a template parameter, chosen per level), and the warp
// walks up it one row at a time, frame rows included.  The phases of a half
// run one row apart in registers: a cell's west / east neighbours are the
// other cell of its pair and, by a shuffle, the nearer cell of the adjacent
// lane's pair; the south / north ones are in the rows the lane already holds.
// Each phase is valid on a frame one cell narrower than the last, so the
// interior is exact.  Input rows are staged kStreamDepth rows ahead in shared
// memory by cp.async, each lane copying its own pair.
//
// The arithmetic is that of the vectorized kernels (stencil4.cuh: q_apply's
// neighbour order west, east, south, north, v_pre2, v_residual, v_restrict,
// v_prolong, v_sweep), which follow the default V-cycle of
// src/solvers/multigrid/cycles.jl:46-77 (ronaldremmerswaal/TwoPhaseAMR.jl).
// Only the order of the coarse right-hand-side and mean sums differs.
#pragma once

#include <cuda_runtime.h>

#include "stencil4.cuh"

namespace tpa {

struct StreamGeom {
    int nbx, nby;  // blocks across / up the level
    int nsx, nsy;  // strips across / up the level
    int rows;      // interior rows of a strip (the kernel's ROWS)
};

constexpr int kStreamWarps = 4;   // warps per CTA
constexpr int kStreamCols = 56;   // interior columns of a strip (32 lanes of column pairs, a 4-cell frame each side)
constexpr int kStreamDepth = 8;   // rows staged ahead
// resident CTAs per SM the kernels are built for: 6 in FP32 (up to 85
// registers), 4 in FP64 (up to 128), which the two-cell rows of the pipeline
// need without spilling
template <typename T>
constexpr int stream_ctas_per_sm() {
    return sizeof(T) == 8 ? 4 : 6;
}

template <int B>
__device__ __forceinline__ void st_cp_async(void* dst, const void* src) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(src), "n"(B) : "memory");
}
__device__ __forceinline__ void st_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void st_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// cell of lattice position (gx, gy), both inside the level
__device__ __forceinline__ int st_cell(const StreamGeom& g, int gx, int gy) {
    return (((gy >> 4) * g.nbx + (gx >> 4)) << 8) + ((gy & 15) << 4) + (gx & 15);
}
// the next level's cell holding fine position (gx, gy) (2 x 2 aggregation)
__device__ __forceinline__ int st_coarse(const StreamGeom& g, int gx, int gy) {
    const int cx = gx >> 1, cy = gy >> 1;
    return (((cy >> 4) * (g.nbx >> 1) + (cx >> 4)) << 8) + ((cy & 15) << 4) + (cx & 15);
}
__device__ __forceinline__ int st_wrap(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// two adjacent cells of a row: the left one at an even column
template <typename T>
struct alignas(2 * sizeof(T)) P2 {
    T l, r;
};

// c0 (4 v - (w + e + s + n)) at the two cells of this lane's pair in a row;
// every lane of the warp calls it (shuffles).  The outer cells of the strip
// get a neighbour of their own pair; their results lie outside the frame that
// is used.
template <typename T>
__device__ __forceinline__ P2<T> st_apply(const SView<T>& L, const P2<T>& s, const P2<T>& c, const P2<T>& n) {
    const T w = __shfl_up_sync(0xffffffffu, c.r, 1);
    const T e = __shfl_down_sync(0xffffffffu, c.l, 1);
    P2<T> o;
    T off = w;
    off += c.r;
    off += s.l;
    off += n.l;
    o.l = L.c0 * (T(4) * c.l - off);
    off = c.l;
    off += e;
    off += s.r;
    off += n.r;
    o.r = L.c0 * (T(4) * c.r - off);
    return o;
}

// Both pre-sweeps from x = 0 with the level's RHS projection, the residual, and
// the restriction b_c = P_tent'(r - wt A D^-1 r) with the optional coarse RHS sum.
// The pre-smoothed iterate goes to L.y and the projected RHS to L.bp (read by
// v_stream_up); the residual stays in registers.  The warps of the grid take the
// strips in turn (the last strip across or up the level may be cut short: its
// cells past the edge are walked but not written).
template <typename T, typename TB, int ROWS>
__global__ void __launch_bounds__(kStreamWarps * 32, stream_ctas_per_sm<T>())
    v_stream_down(SView<T> L, StreamGeom g, const TB* __restrict__ bin, const double* level_sum,
                  T* __restrict__ bc, double* partial, unsigned* counter, double* coarse_sum) {
    pdl_entry();
    constexpr int S = ROWS + 6, D = kStreamDepth;
    __shared__ P2<TB> stage[kStreamWarps][D][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int W = g.nbx * 16, H = g.nby * 16;
    const double mean = (L.singular && level_sum) ? *level_sum * L.cvol_inv : 0.0;
    const double vol0 = double(L.vol0);
    const T wd = L.w * L.dinv0;
    auto proj = [&](TB a) { return mean != 0.0 ? T(double(a) - vol0 * mean) : T(a); };
    double part = 0;
    for (int strip = blockIdx.x * kStreamWarps + wid; strip < g.nsx * g.nsy; strip += gridDim.x * kStreamWarps) {
        const int x0 = (strip % g.nsx) * kStreamCols, y0 = (strip / g.nsx) * ROWS;
        const int gx0 = x0 - 4 + 2 * lane;
        const bool out_col = lane >= 2 && lane < 2 + kStreamCols / 2 && gx0 < W;
        const int gx = st_wrap(gx0, W);
        auto cell = [&](int k) { return st_cell(g, gx, st_wrap(y0 - 3 + k, H)); };
        auto in_row = [&](int j) { return y0 + j - 3 < H; };  // interior row j inside the level
#pragma unroll
        for (int k = 0; k < D - 1; ++k) {
            st_cp_async<sizeof(P2<TB>)>(&stage[wid][k][lane], bin + cell(k));
            st_commit();
        }
        P2<T> bp[S], x1[S], x2[S], r[S], s[S], t[S];
#pragma unroll
        for (int k = 0; k < S; ++k) {
            if (k + D - 1 < S) st_cp_async<sizeof(P2<TB>)>(&stage[wid][(k + D - 1) % D][lane], bin + cell(k + D - 1));
            st_commit();
            st_wait<D - 1>();
            const P2<TB> a = stage[wid][k % D][lane];
            bp[k] = P2<T>{proj(a.l), proj(a.r)};
            x1[k] = P2<T>{wd * bp[k].l, wd * bp[k].r};  // the first sweep from zero, pointwise
            if (k >= 2) {  // rows 1 .. S - 2
                const int j = k - 1;
                const P2<T> ax = st_apply(L, x1[j - 1], x1[j], x1[j + 1]);
                x2[j] = P2<T>{x1[j].l + wd * (bp[j].l - ax.l), x1[j].r + wd * (bp[j].r - ax.r)};
                if (j >= 3 && j < 3 + ROWS && out_col && in_row(j)) {
                    const int c = cell(j);
                    *reinterpret_cast<P2<T>*>(L.y + c) = x2[j];
                    *reinterpret_cast<P2<T>*>(L.bp + c) = bp[j];
                }
            }
            if (k >= 4) {  // rows 2 .. S - 3: their x2 neighbours exist
                const int j = k - 2;
                const P2<T> ax = st_apply(L, x2[j - 1], x2[j], x2[j + 1]);
                r[j] = P2<T>{bp[j].l - ax.l, bp[j].r - ax.r};
                s[j] = P2<T>{L.dinv0 * r[j].l, L.dinv0 * r[j].r};
            }
            if (k >= 6) {  // rows 3 .. S - 4: the interior
                const int j = k - 3;
                const P2<T> as = st_apply(L, s[j - 1], s[j], s[j + 1]);
                t[j] = P2<T>{r[j].l - L.tw * as.l, r[j].r - L.tw * as.r};
                // rows j - 1 and j of the interior are a coarse row: the pair of
                // each row, then the row above, as v_restrict sums them
                if (j >= 4 && j < 3 + ROWS && (j & 1) == 0 && out_col && in_row(j)) {
                    const T h0 = t[j - 1].l + t[j - 1].r;
                    const T d0 = t[j].l + t[j].r;
                    const T v = h0 + d0;
                    bc[st_coarse(g, gx, y0 + j - 4)] = v;
                    part += double(v);
                }
            }
        }
    }
    if (coarse_sum) {
        if (publish_partial(part, partial, counter)) {
            const double sum = fold_partials(partial, gridDim.x);
            if (threadIdx.x == 0) {
                *coarse_sum = sum;
                *counter = 0;
            }
        }
    }
}

// The prolongation x = y + e - wt D^-1 A e with e = P_tent x_c (y: the
// pre-smoothed iterate of v_stream_down; both cells of a pair share their
// coarse cell) and both post-sweeps into L.x; with `mean_out`, the volume mean
// of L.x (and the epilogue's sums) folded.
template <typename T, typename Epi, int ROWS>
__global__ void __launch_bounds__(kStreamWarps * 32, stream_ctas_per_sm<T>())
    v_stream_up(SView<T> L, StreamGeom g, const T* __restrict__ xc, double* partial, unsigned* counter,
                double* mean_out, Epi epi) {
    pdl_entry();
    constexpr int S = ROWS + 6, D = kStreamDepth;
    __shared__ T se[kStreamWarps][D][32];
    __shared__ P2<T> sy[kStreamWarps][D][32], sb[kStreamWarps][D][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int W = g.nbx * 16, H = g.nby * 16;
    const T wd = L.w * L.dinv0;
    double v = 0, w = 0;
    for (int strip = blockIdx.x * kStreamWarps + wid; strip < g.nsx * g.nsy; strip += gridDim.x * kStreamWarps) {
        const int x0 = (strip % g.nsx) * kStreamCols, y0 = (strip / g.nsx) * ROWS;
        const int gx0 = x0 - 4 + 2 * lane;
        const bool out_col = lane >= 2 && lane < 2 + kStreamCols / 2 && gx0 < W;
        const int gx = st_wrap(gx0, W);
        auto stage_row = [&](int k) {
            const int gy = st_wrap(y0 - 3 + k, H);
            const int c = st_cell(g, gx, gy);
            st_cp_async<sizeof(T)>(&se[wid][k % D][lane], xc + st_coarse(g, gx, gy));
            st_cp_async<sizeof(P2<T>)>(&sy[wid][k % D][lane], L.y + c);
            st_cp_async<sizeof(P2<T>)>(&sb[wid][k % D][lane], L.bp + c);
        };
#pragma unroll
        for (int k = 0; k < D - 1; ++k) {
            stage_row(k);
            st_commit();
        }
        P2<T> e[S], y[S], b[S], p[S], q[S];
#pragma unroll
        for (int k = 0; k < S; ++k) {
            if (k + D - 1 < S) stage_row(k + D - 1);
            st_commit();
            st_wait<D - 1>();
            const T ek = se[wid][k % D][lane];
            e[k] = P2<T>{ek, ek};
            y[k] = sy[wid][k % D][lane];
            b[k] = sb[wid][k % D][lane];
            if (k >= 2) {  // rows 1 .. S - 2
                const int j = k - 1;
                const P2<T> ae = st_apply(L, e[j - 1], e[j], e[j + 1]);
                p[j] = P2<T>{y[j].l + (e[j].l - L.tw * L.dinv0 * ae.l), y[j].r + (e[j].r - L.tw * L.dinv0 * ae.r)};
            }
            if (k >= 4) {  // rows 2 .. S - 3
                const int j = k - 2;
                const P2<T> ap = st_apply(L, p[j - 1], p[j], p[j + 1]);
                q[j] = P2<T>{p[j].l + wd * (b[j].l - ap.l), p[j].r + wd * (b[j].r - ap.r)};
            }
            if (k >= 6) {  // rows 3 .. S - 4: the interior
                const int j = k - 3;
                const P2<T> aq = st_apply(L, q[j - 1], q[j], q[j + 1]);
                const P2<T> o{q[j].l + wd * (b[j].l - aq.l), q[j].r + wd * (b[j].r - aq.r)};
                if (j >= 3 && j < 3 + ROWS && out_col && y0 + j - 3 < H) {
                    const int c = st_cell(g, gx, y0 + j - 3);
                    *reinterpret_cast<P2<T>*>(L.x + c) = o;
                    if (mean_out) {
                        v += double(L.vol0) * double(o.l);
                        v += double(L.vol0) * double(o.r);
                        if constexpr (Epi::kRz) {
                            w += epi.r[c] * double(o.l);
                            w += epi.r[c + 1] * double(o.r);
                        }
                    }
                }
            }
        }
    }
    if (mean_out) fold_mean(v, w, partial, counter, mean_out, L.cvol_inv, epi);
}

}  // namespace tpa
