// Inverse face metric K (the face Riesz map of the pressure gradient).
//
// Reproduces (ronaldremmerswaal/TwoPhaseAMR.jl):
//   src/operators/gradient.jl:107-158  face displacement from integer lattice offsets
//   src/operators/gradient.jl:160-171  vertex keys of face endpoints (periodic wrap)
//   src/operators/gradient.jl:194-232  dense vertex-patch metric: symmetrised moment
//                                      tensor, consistent part + trace/(n-2) projector
//   src/operators/gradient.jl:234-267  template cache keyed by scale-normalised
//                                      descriptors (faces sorted by descriptor)
//   src/operators/gradient.jl:269-292  physical-wall / two-face patches: half of the
//                                      two-point metric per endpoint
//   src/operators/gradient.jl:294-367  endpoint order (x, then y, then endpoint),
//                                      duplicate entries summed, zeros dropped
#include <algorithm>
#include <cmath>
#include <map>

#include "host.hpp"

namespace tpa {
namespace {

// Solve the 2x2 system A X = B (B: 2 x n, column-major per column) with partial
// pivoting, in place on B.
void solve2(const double A_in[2][2], double* B, int ncols) {
    double a00 = A_in[0][0], a01 = A_in[0][1], a10 = A_in[1][0], a11 = A_in[1][1];
    bool swap = std::fabs(a10) > std::fabs(a00);
    if (swap) { std::swap(a00, a10); std::swap(a01, a11); }
    double l10 = a10 / a00;
    double u11 = a11 - l10 * a01;
    for (int c = 0; c < ncols; ++c) {
        double b0 = B[2 * c], b1 = B[2 * c + 1];
        if (swap) std::swap(b0, b1);
        b1 = b1 - l10 * b0;
        double x1 = b1 / u11;
        double x0 = (b0 - a01 * x1) / a00;
        B[2 * c] = x0;
        B[2 * c + 1] = x1;
    }
}

struct PatchFace {
    int32_t index;
    int axis;
    double area, dx, dy;
};

// Dense symmetric local metric of one interior vertex patch (row-major n x n).
std::vector<double> local_metric(const std::vector<PatchFace>& faces) {
    const int n = int(faces.size());
    if (n <= 2) throw Error(1, "a periodic vertex patch must contain at least three faces");
    std::vector<double> M(static_cast<size_t>(2 * n)), N(static_cast<size_t>(2 * n), 0.0);  // row-major n x 2
    for (int r = 0; r < n; ++r) {
        M[size_t(2 * r)] = faces[size_t(r)].area * faces[size_t(r)].dx;
        M[size_t(2 * r + 1)] = faces[size_t(r)].area * faces[size_t(r)].dy;
        N[size_t(2 * r + faces[size_t(r)].axis - 1)] = 0.5;
    }
    double mn[2][2] = {{0, 0}, {0, 0}}, gram[2][2] = {{0, 0}, {0, 0}};
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int r = 0; r < n; ++r) {
                mn[a][b] += M[size_t(2 * r + a)] * N[size_t(2 * r + b)];
                gram[a][b] += M[size_t(2 * r + a)] * M[size_t(2 * r + b)];
            }
    double s01 = (mn[0][1] + mn[1][0]) / 2;
    mn[0][1] = mn[1][0] = s01;
    if (!(mn[0][0] > 0 && mn[0][0] * mn[1][1] - mn[0][1] * mn[1][0] > 0))
        throw Error(1, "degenerate vertex patch in gradient construction");
    std::vector<double> X(static_cast<size_t>(2 * n)), Y(static_cast<size_t>(2 * n));  // column c = (x0, x1)
    for (int c = 0; c < n; ++c) {
        X[size_t(2 * c)] = N[size_t(2 * c)];
        X[size_t(2 * c + 1)] = N[size_t(2 * c + 1)];
        Y[size_t(2 * c)] = M[size_t(2 * c)];
        Y[size_t(2 * c + 1)] = M[size_t(2 * c + 1)];
    }
    solve2(mn, X.data(), n);    // mn \ N'
    solve2(gram, Y.data(), n);  // gram \ M'
    std::vector<double> L(static_cast<size_t>(n * n));
    double trace = 0;
    for (int r = 0; r < n; ++r)
        trace += N[size_t(2 * r)] * X[size_t(2 * r)] + N[size_t(2 * r + 1)] * X[size_t(2 * r + 1)];
    const double stab = trace / double(n - 2);
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            double consistent = N[size_t(2 * r)] * X[size_t(2 * c)] + N[size_t(2 * r + 1)] * X[size_t(2 * c + 1)];
            double proj = (r == c ? 1.0 : 0.0) -
                          (M[size_t(2 * r)] * Y[size_t(2 * c)] + M[size_t(2 * r + 1)] * Y[size_t(2 * c + 1)]);
            L[size_t(r * n + c)] = consistent + stab * proj;
        }
    std::vector<double> S(static_cast<size_t>(n * n));
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) S[size_t(r * n + c)] = (L[size_t(r * n + c)] + L[size_t(c * n + r)]) / 2;
    return S;
}

}  // namespace

Metric assemble_metric(const Mesh& m) {
    const int64_t nf = m.nfaces();
    int64_t lat[2];
    m.lattice(m.active, lat);
    Metric K;
    K.diag.assign(static_cast<size_t>(nf), 0.0);
    std::vector<double> dx(static_cast<size_t>(nf)), dy(static_cast<size_t>(nf));
    std::vector<int64_t> ex(static_cast<size_t>(2 * nf)), ey(static_cast<size_t>(2 * nf));
    const int64_t cpb = m.cells_per_block();
    for (int64_t f = 0; f < nf; ++f) {
        int64_t ml[2], ms[2], pl[2], ps[2];
        m.cell_lattice(m.fm[size_t(f)], lat, ml, ms);
        m.cell_lattice(m.fp[size_t(f)], lat, pl, ps);
        int a = m.fax[size_t(f)] - 1, t = 1 - a;
        int64_t bm = m.fm[size_t(f)] / cpb, bp = m.fp[size_t(f)] / cpb;
        double hm = a == 0 ? m.bsx[size_t(bm)] : m.bsy[size_t(bm)];
        double hp = a == 0 ? m.bsx[size_t(bp)] : m.bsy[size_t(bp)];
        double normal = (hm + hp) / 2;
        int64_t offset = 2 * pl[t] + ps[t] - 2 * ml[t] - ms[t];
        if (m.periodic[t]) {
            if (offset > lat[t]) offset -= 2 * lat[t];
            if (offset < -lat[t]) offset += 2 * lat[t];
        }
        double tangential = double(offset) * ((m.extent[t] / double(lat[t])) / 2);
        dx[size_t(f)] = a == 0 ? normal : tangential;
        dy[size_t(f)] = a == 0 ? tangential : normal;
        int64_t nrm, lo, hi;
        m.face_lattice(f, lat, nrm, lo, hi);
        for (int e = 0; e < 2; ++e) {
            int64_t tang = e == 0 ? lo : hi;
            int64_t vi = a == 0 ? nrm : tang, vj = a == 0 ? tang : nrm;
            if (m.periodic[0]) vi = ((vi % lat[0]) + lat[0]) % lat[0];
            if (m.periodic[1]) vj = ((vj % lat[1]) + lat[1]) % lat[1];
            ex[size_t(2 * f + e)] = vi;
            ey[size_t(2 * f + e)] = vj;
        }
    }
    // Two stable counting sorts: by y, then by x.
    const int64_t ne = 2 * nf;
    std::vector<int64_t> by_y(static_cast<size_t>(ne)), order(static_cast<size_t>(ne));
    {
        std::vector<int64_t> cnt(static_cast<size_t>(lat[1] + 2), 0);
        for (int64_t e = 0; e < ne; ++e) cnt[size_t(ey[size_t(e)] + 1)]++;
        for (int64_t k = 0; k <= lat[1]; ++k) cnt[size_t(k + 1)] += cnt[size_t(k)];
        for (int64_t e = 0; e < ne; ++e) by_y[size_t(cnt[size_t(ey[size_t(e)])]++)] = e;
        std::vector<int64_t> cx(static_cast<size_t>(lat[0] + 2), 0);
        for (int64_t e = 0; e < ne; ++e) cx[size_t(ex[size_t(e)] + 1)]++;
        for (int64_t k = 0; k <= lat[0]; ++k) cx[size_t(k + 1)] += cx[size_t(k)];
        for (int64_t p = 0; p < ne; ++p) {
            int64_t e = by_y[size_t(p)];
            order[size_t(cx[size_t(ex[size_t(e)])]++)] = e;
        }
    }
    std::map<std::vector<std::array<double, 4>>, std::vector<double>> cache;
    struct Trip { int32_t r, c; double v; };
    std::vector<Trip> off;
    std::vector<PatchFace> faces;
    std::vector<std::array<double, 4>> desc;
    int64_t pos = 0;
    while (pos < ne) {
        int64_t stop = pos + 1;
        const int64_t x = ex[size_t(order[size_t(pos)])], y = ey[size_t(order[size_t(pos)])];
        while (stop < ne && ex[size_t(order[size_t(stop)])] == x && ey[size_t(order[size_t(stop)])] == y) ++stop;
        faces.clear();
        for (int64_t p = pos; p < stop; ++p) {
            int32_t f = int32_t(order[size_t(p)] >> 1);
            faces.push_back({f, m.fax[size_t(f)], m.farea[size_t(f)], dx[size_t(f)], dy[size_t(f)]});
        }
        pos = stop;
        bool physical = (!m.periodic[0] && (x == 0 || x == lat[0])) || (!m.periodic[1] && (y == 0 || y == lat[1]));
        if (physical || faces.size() <= 2) {
            for (const auto& pf : faces) {
                double nd = std::fabs(pf.axis == 1 ? pf.dx : pf.dy);
                if (!(nd > 0)) throw Error(1, "degenerate face beside a physical boundary");
                K.diag[size_t(pf.index)] += 1.0 / (2.0 * pf.area * nd);
            }
            continue;
        }
        double scale = 0;
        for (const auto& pf : faces) scale = std::max(scale, std::max(pf.area, std::max(std::fabs(pf.dx), std::fabs(pf.dy))));
        if (!(scale > 0)) throw Error(1, "degenerate vertex-patch scale");
        auto descriptor = [&](const PatchFace& pf) {
            return std::array<double, 4>{double(pf.axis), pf.area / scale, pf.dx / scale, pf.dy / scale};
        };
        std::stable_sort(faces.begin(), faces.end(),
                         [&](const PatchFace& u, const PatchFace& v) { return descriptor(u) < descriptor(v); });
        desc.clear();
        for (const auto& pf : faces) desc.push_back(descriptor(pf));
        auto it = cache.find(desc);
        if (it == cache.end()) {
            std::vector<double> L = local_metric(faces);
            for (auto& v : L) v *= scale * scale;
            it = cache.emplace(desc, std::move(L)).first;
        }
        const std::vector<double>& normalized = it->second;
        const int n = int(faces.size());
        for (int c = 0; c < n; ++c)
            for (int r = 0; r < n; ++r) {
                double v = normalized[size_t(r * n + c)] / (scale * scale);
                int32_t fr = faces[size_t(r)].index, fc = faces[size_t(c)].index;
                if (fr == fc) K.diag[size_t(fr)] += v;
                else if (v != 0.0) off.push_back({fr, fc, v});
            }
    }
    K.templates = int(cache.size());
    std::stable_sort(off.begin(), off.end(), [](const Trip& u, const Trip& v) {
        return u.c != v.c ? u.c < v.c : u.r < v.r;
    });
    for (size_t k = 0; k < off.size();) {
        size_t e = k;
        double s = 0.0;
        bool first = true;
        while (e < off.size() && off[e].r == off[k].r && off[e].c == off[k].c) {
            s = first ? off[e].v : s + off[e].v;
            first = false;
            ++e;
        }
        if (s != 0.0) {
            K.off_row.push_back(off[k].r);
            K.off_col.push_back(off[k].c);
            K.off_val.push_back(s);
        }
        k = e;
    }
    for (double d : K.diag)
        if (!(d > 0)) throw Error(1, "gradient Riesz map has a non-positive diagonal");
    return K;
}

}  // namespace tpa
