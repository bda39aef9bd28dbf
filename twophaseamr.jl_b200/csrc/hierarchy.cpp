// Assembled level operators and the rediscretised tree hierarchy.
//
// Reproduces (ronaldremmerswaal/TwoPhaseAMR.jl):
//   src/operators/elliptic.jl:157-257   symmetric stiffness (A + A')/2 of J' M J with
//                                       M = k K (diagonal K) or sqrt(k) K sqrt(k)
//   src/solvers/multigrid/elliptic_solver.jl:1-129, two_phase/projection/common.jl:53-83
//                                       open-face components; a component touching an open
//                                       (Dirichlet) side is anchored, the others ungauged
//   src/operators/elliptic.jl:76-152, 757-764   open sides: boundary material, the
//                                       conductance 2 k_b / h |f| added to the diagonal
//   src/solvers/multigrid/hierarchy.jl:8-30        `_jacobi_weight!`
//   src/solvers/multigrid/hierarchy.jl:631-721     smoothed transfer weights
//   src/solvers/multigrid/hierarchy.jl:786-817     `_multigrid_level` (row sums, weight)
//   src/solvers/multigrid/tree_coarsening.jl:30-82, 187-212  coarse meshes and stopping
//   src/solvers/multigrid/tree_coarsening.jl:228-252         tentative owners
//   src/solvers/multigrid/tree_coarsening.jl:347-398, 538-555 face-coefficient restriction
//   src/solvers/multigrid/geometric_preconditioner.jl:144-169, 420-430  augmented coarse solve
#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>
#include <tuple>

#include "host.hpp"

namespace tpa {

double Csr::diag(int64_t r) const {
    for (int64_t k = ptr[size_t(r)]; k < ptr[size_t(r + 1)]; ++k)
        if (col[size_t(k)] == r) return val[size_t(k)];
    return 0.0;
}

namespace {

int32_t find_root(std::vector<int32_t>& parent, int32_t x) {
    while (parent[size_t(x)] != x) {
        parent[size_t(x)] = parent[size_t(parent[size_t(x)])];
        x = parent[size_t(x)];
    }
    return x;
}

// `_elliptic_boundary_data!` (elliptic.jl:136-152) with unit apertures and
// no inactive cells: the gradient factor 2 k_b / h of every open boundary face
// and the diagonal term |f| times it of its cell
void boundary_data(LevelOperator& op) {
    const Mesh& m = op.mesh;
    const int64_t nb = int64_t(m.bcell.size());
    op.bdiag.clear();
    op.bgrad.assign(size_t(nb), 0.0);
    if (!op.any_open()) return;
    if (int64_t(op.bkappa.size()) != nb) throw Error(1, "one coefficient is required per boundary face");
    op.bdiag.assign(size_t(m.ncells()), 0.0);
    const int64_t cpb = m.cells_per_block();
    for (int64_t b = 0; b < nb; ++b) {
        if (!op.open_face(b)) continue;
        const int32_t cell = m.bcell[size_t(b)];
        if (!(op.volumes[size_t(cell)] > 0)) continue;
        const int64_t blk = cell / cpb;
        const double h = m.bax[size_t(b)] == 1 ? m.bsx[size_t(blk)] : m.bsy[size_t(blk)];
        const double factor = 2 * op.bkappa[size_t(b)] / h;
        op.bgrad[size_t(b)] = factor;
        op.bdiag[size_t(cell)] += m.barea[size_t(b)] * factor;
    }
}

Components components(const LevelOperator& op) {
    const Mesh& m = op.mesh;
    const int64_t nc = m.ncells();
    std::vector<int32_t> parent(static_cast<size_t>(nc));
    std::iota(parent.begin(), parent.end(), 0);
    for (int64_t f = 0; f < m.nfaces(); ++f) {
        if (op.kappa[size_t(f)] == 0.0) continue;
        int32_t a = find_root(parent, m.fm[size_t(f)]), b = find_root(parent, m.fp[size_t(f)]);
        if (a != b) parent[size_t(std::max(a, b))] = std::min(a, b);  // root = smallest cell
    }
    Components c;
    c.slot.assign(static_cast<size_t>(nc), -1);
    std::vector<int32_t> root_slot(static_cast<size_t>(nc), -1);
    // a cell with an open-face conductance anchors its component
    // (elliptic_solver.jl:80-82)
    std::vector<char> anchored(static_cast<size_t>(nc), 0);
    for (size_t i = 0; i < op.bdiag.size(); ++i)
        if (op.bdiag[i] != 0.0) anchored[size_t(find_root(parent, int32_t(i)))] = 1;
    for (int64_t i = 0; i < nc; ++i) {
        if (!(op.volumes[size_t(i)] > 0)) continue;
        int32_t r = find_root(parent, int32_t(i));
        if (anchored[size_t(r)]) continue;
        if (root_slot[size_t(r)] < 0) {
            root_slot[size_t(r)] = int32_t(c.anchor.size());
            c.anchor.push_back(r);
            c.volume.push_back(0.0);
        }
        c.slot[size_t(i)] = root_slot[size_t(r)];
        c.volume[size_t(root_slot[size_t(r)])] += op.volumes[size_t(i)];
    }
    return c;
}

}  // namespace

bool LevelOperator::open_face(int64_t b) const {
    return open[2 * (mesh.bax[size_t(b)] - 1) + (mesh.bside[size_t(b)] > 0 ? 1 : 0)];
}

void extend_boundary_material(LevelOperator& op) {
    const Mesh& m = op.mesh;
    const int64_t nb = int64_t(m.bcell.size());
    op.bkappa.assign(size_t(nb), 0.0);
    if (!op.any_open()) return;
    if (int64_t(op.kappa.size()) != m.nfaces()) throw Error(1, "one coefficient is required per interior face");
    std::map<std::tuple<int32_t, int, int>, int64_t> index;
    for (int64_t b = 0; b < nb; ++b)
        if (op.open_face(b)) index[{m.bcell[size_t(b)], int(m.bax[size_t(b)]), int(m.bside[size_t(b)])}] = b;
    std::vector<double> weights(size_t(nb), 0.0);
    for (int64_t f = 0; f < m.nfaces(); ++f) {
        const std::pair<int32_t, int> ends[2] = {{m.fm[size_t(f)], -1}, {m.fp[size_t(f)], 1}};
        for (const auto& [cell, side] : ends) {
            auto it = index.find({cell, int(m.fax[size_t(f)]), side});
            if (it == index.end()) continue;
            op.bkappa[size_t(it->second)] += m.farea[size_t(f)] * op.kappa[size_t(f)];
            weights[size_t(it->second)] += m.farea[size_t(f)];
        }
    }
    for (const auto& [key, b] : index) {
        if (!(weights[size_t(b)] > 0))
            throw Error(1, "cannot extend an interior coefficient to an open face without an opposite interior "
                           "face; supply boundary face coefficients");
        op.bkappa[size_t(b)] /= weights[size_t(b)];
    }
}

void assemble_operator(LevelOperator& op) {
    const Mesh& m = op.mesh;
    const int64_t nc = m.ncells(), nf = m.nfaces();
    if (int64_t(op.kappa.size()) != nf) throw Error(1, "one coefficient is required per interior face");
    for (double k : op.kappa)
        if (!std::isfinite(k) || k < 0) throw Error(1, "face coefficients must be finite and nonnegative");
    op.volumes = m.cell_volumes();
    const Metric& K = op.metric;
    const bool diagonal = K.diagonal();
    std::vector<int64_t> cnt(static_cast<size_t>(nc + 1), 0);
    for (int64_t f = 0; f < nf; ++f) {
        cnt[size_t(m.fm[size_t(f)]) + 1] += 2;
        cnt[size_t(m.fp[size_t(f)]) + 1] += 2;
    }
    for (size_t k = 0; k < K.off_val.size(); ++k) {
        cnt[size_t(m.fm[size_t(K.off_row[k])]) + 1] += 2;
        cnt[size_t(m.fp[size_t(K.off_row[k])]) + 1] += 2;
    }
    for (int64_t c = 0; c < nc; ++c) cnt[size_t(c + 1)] += cnt[size_t(c)];
    std::vector<int64_t> next(cnt.begin(), cnt.end() - 1);
    std::vector<std::pair<int32_t, double>> raw(static_cast<size_t>(cnt[size_t(nc)]));
    auto add = [&](int32_t r, int32_t c, double v) { raw[size_t(next[size_t(r)]++)] = {c, v}; };
    std::vector<double> sk(static_cast<size_t>(nf));
    for (int64_t f = 0; f < nf; ++f) sk[size_t(f)] = std::sqrt(op.kappa[size_t(f)]);
    for (int64_t f = 0; f < nf; ++f) {
        double kf = K.diag[size_t(f)];
        double w = diagonal ? op.kappa[size_t(f)] * kf : (sk[size_t(f)] * kf) * sk[size_t(f)];
        double a = m.farea[size_t(f)];
        int32_t cm = m.fm[size_t(f)], cp = m.fp[size_t(f)];
        add(cm, cm, (-a * w) * -a);
        add(cm, cp, (-a * w) * a);
        add(cp, cm, (a * w) * -a);
        add(cp, cp, (a * w) * a);
    }
    for (size_t k = 0; k < K.off_val.size(); ++k) {
        int32_t l = K.off_row[k], r = K.off_col[k];
        double w = (sk[size_t(l)] * K.off_val[k]) * sk[size_t(r)];
        double al = m.farea[size_t(l)], ar = m.farea[size_t(r)];
        int32_t lc[2] = {m.fm[size_t(l)], m.fp[size_t(l)]}, rc[2] = {m.fm[size_t(r)], m.fp[size_t(r)]};
        double ls[2] = {-al, al}, rs[2] = {-ar, ar};
        for (int u = 0; u < 2; ++u)
            for (int v = 0; v < 2; ++v) add(lc[u], rc[v], (ls[u] * w) * rs[v]);
    }
    Csr A;
    A.n = nc;
    A.ptr.assign(static_cast<size_t>(nc + 1), 0);
    std::vector<std::pair<int32_t, double>> row;
    for (int64_t r = 0; r < nc; ++r) {
        row.assign(raw.begin() + cnt[size_t(r)], raw.begin() + cnt[size_t(r + 1)]);
        std::stable_sort(row.begin(), row.end(), [](auto& x, auto& y) { return x.first < y.first; });
        bool has_diag = false;
        for (size_t k = 0; k < row.size();) {
            size_t e = k;
            double s = row[k].second;
            for (++e; e < row.size() && row[e].first == row[k].first; ++e) s += row[e].second;
            if (row[k].first == r) has_diag = true;
            A.col.push_back(row[k].first);
            A.val.push_back(s);
            k = e;
        }
        if (!has_diag) {  // isolated cell: explicit zero diagonal
            auto pos = std::lower_bound(A.col.begin() + A.ptr[size_t(r)], A.col.end(), int32_t(r));
            size_t at = size_t(pos - A.col.begin());
            A.col.insert(A.col.begin() + long(at), int32_t(r));
            A.val.insert(A.val.begin() + long(at), 0.0);
        }
        A.ptr[size_t(r + 1)] = int64_t(A.col.size());
    }
    // symmetric average (A + A')/2 on the (structurally symmetric) pattern
    std::vector<double> sym(A.val.size());
    for (int64_t r = 0; r < nc; ++r)
        for (int64_t k = A.ptr[size_t(r)]; k < A.ptr[size_t(r + 1)]; ++k) {
            int32_t c = A.col[size_t(k)];
            auto b = A.col.begin() + A.ptr[size_t(c)], e = A.col.begin() + A.ptr[size_t(c + 1)];
            auto it = std::lower_bound(b, e, int32_t(r));
            if (it == e || *it != r) throw Error(1, "sparse topology is missing a required entry");
            double v = (A.val[size_t(k)] + A.val[size_t(it - A.col.begin())]) / 2;
            sym[size_t(k)] = v == 0.0 ? 0.0 : v;
        }
    A.val.swap(sym);
    // open-face conductances on the diagonal, after the symmetric average
    // (elliptic.jl:757-764)
    boundary_data(op);
    for (size_t r = 0; r < op.bdiag.size(); ++r) {
        if (op.bdiag[r] == 0.0) continue;
        for (int64_t k = A.ptr[r]; k < A.ptr[r + 1]; ++k)
            if (A.col[size_t(k)] == int32_t(r)) A.val[size_t(k)] += op.bdiag[r];
    }
    op.A = std::move(A);
    op.comp = components(op);
    op.singular = !op.comp.anchor.empty();
}

double jacobi_weight(std::vector<double>& inv, const std::vector<double>& rs, bool skip_nonpositive,
                     bool allow_zero, bool clamp, double zero_weight) {
    double bound = 0.0;
    for (size_t k = 0; k < inv.size(); ++k) {
        double d = inv[k];
        if (d == 0.0 && allow_zero) continue;
        if (!(d > 0)) {
            if (skip_nonpositive) continue;
            throw Error(1, "elliptic matrix has a non-positive diagonal");
        }
        bound = std::max(bound, rs[k] / d);
        inv[k] = 1.0 / d;
    }
    if (bound == 0.0) return zero_weight;
    double w = 4.0 / (3.0 * bound);
    return clamp ? std::min(1.0, w) : w;
}

namespace {

void diag_and_rowsums(const Csr& A, std::vector<double>& d, std::vector<double>& rs) {
    d.assign(static_cast<size_t>(A.n), 0.0);
    rs.assign(static_cast<size_t>(A.n), 0.0);
    for (int64_t r = 0; r < A.n; ++r)
        for (int64_t k = A.ptr[size_t(r)]; k < A.ptr[size_t(r + 1)]; ++k) {
            rs[size_t(r)] += std::fabs(A.val[size_t(k)]);
            if (A.col[size_t(k)] == r) d[size_t(r)] = A.val[size_t(k)];
        }
}

bool coarsened_base(const Mesh& m, Mesh& out) {
    const Forest& f = m.forest;
    if (f.layout[0] % 2 || f.layout[1] % 2) return false;
    int base[2] = {m.base[0] / 2, m.base[1] / 2};
    for (int a = 0; a < 2; ++a)
        if (m.periodic[a] && base[a] < 4) return false;
    Forest g;
    for (int a = 0; a < 2; ++a) {
        g.layout[a] = f.layout[a] / 2;
        g.origin[a] = m.origin[a];
        g.extent[a] = m.extent[a];
        g.root_extent[a] = m.extent[a] / g.layout[a];
    }
    for (int j = 0; j < g.layout[1]; ++j)
        for (int i = 0; i < g.layout[0]; ++i) g.leaves.insert(pack_key(0, i, j));
    out = mesh_from_forest(std::move(g), base, m.bs, m.periodic);
    return true;
}

Mesh pruned(const Mesh& m) {
    const Forest& f = m.forest;
    Forest g;
    for (int a = 0; a < 2; ++a) {
        g.layout[a] = f.layout[a];
        g.origin[a] = f.origin[a];
        g.extent[a] = f.extent[a];
        g.root_extent[a] = f.root_extent[a];
    }
    for (uint64_t n : f.internal) {
        int lev = key_level(n);
        bool keep = false;
        for (int cj = 0; cj < 2 && !keep; ++cj)
            for (int ci = 0; ci < 2 && !keep; ++ci)
                keep = f.internal.count(pack_key(lev + 1, 2 * key_i(n) + ci, 2 * key_j(n) + cj)) > 0;
        if (keep) g.internal.insert(n);
    }
    for (int j = 0; j < g.layout[1]; ++j)
        for (int i = 0; i < g.layout[0]; ++i)
            if (!g.internal.count(pack_key(0, i, j))) g.leaves.insert(pack_key(0, i, j));
    for (uint64_t n : g.internal) {
        int lev = key_level(n);
        for (int cj = 0; cj < 2; ++cj)
            for (int ci = 0; ci < 2; ++ci) {
                uint64_t c = pack_key(lev + 1, 2 * key_i(n) + ci, 2 * key_j(n) + cj);
                if (!g.internal.count(c)) g.leaves.insert(c);
            }
    }
    g.balance(m.periodic);
    return mesh_from_forest(std::move(g), m.base, m.bs, m.periodic);
}

bool next_coarse(const Mesh& cur, const HierarchyOptions& o, int nlevels, Mesh& out) {
    if (!(cur.ncells() > o.coarse_size && nlevels < o.max_levels)) return false;
    if (cur.active == 0) {
        if (!coarsened_base(cur, out)) return false;
    } else {
        out = pruned(cur);
    }
    return out.ncells() < cur.ncells();
}

std::vector<int32_t> owners(const Mesh& fine, const Mesh& coarse) {
    int64_t lf[2], lc[2], lat[2];
    fine.lattice(fine.active, lf);
    coarse.lattice(coarse.active, lc);
    lat[0] = std::max(lf[0], lc[0]);
    lat[1] = std::max(lf[1], lc[1]);
    const Forest& t = coarse.forest;
    int64_t root_w[2] = {lat[0] / t.layout[0], lat[1] / t.layout[1]};
    const int nx = coarse.bs[0], ny = coarse.bs[1];
    std::vector<int32_t> own(static_cast<size_t>(fine.ncells()));
    for (int64_t c = 0; c < fine.ncells(); ++c) {
        int64_t low[2], sc[2];
        fine.cell_lattice(c, lat, low, sc);
        int64_t x = low[0] + sc[0] / 2, y = low[1] + sc[1] / 2;
        uint64_t key = pack_key(0, x / root_w[0], y / root_w[1]);
        while (!t.leaves.count(key)) {
            int lev = key_level(key) + 1;
            key = pack_key(lev, x / (root_w[0] >> lev), y / (root_w[1] >> lev));
        }
        int lev = key_level(key);
        int64_t s0 = lat[0] / ((int64_t(t.layout[0]) * nx) << lev), s1 = lat[1] / ((int64_t(t.layout[1]) * ny) << lev);
        int64_t ci = (x / s0) % nx, cj = (y / s1) % ny;
        own[size_t(c)] = int32_t(int64_t(coarse.index.at(key)) * nx * ny + cj * nx + ci);
    }
    return own;
}

void face_restriction(const Mesh& coarse, const Mesh& fine, std::vector<int64_t>& ptr, std::vector<int32_t>& idx,
                      std::vector<double>& w, bool boundary = false) {
    int64_t lf[2], lc[2], lat[2];
    fine.lattice(fine.active, lf);
    coarse.lattice(coarse.active, lc);
    lat[0] = std::max(lf[0], lc[0]);
    lat[1] = std::max(lf[1], lc[1]);
    struct Seg { int64_t lo, hi; int32_t f; };
    std::map<std::pair<int, int64_t>, std::vector<Seg>> lines;
    const int64_t nfine = boundary ? int64_t(fine.bcell.size()) : fine.nfaces();
    for (int64_t f = 0; f < nfine; ++f) {
        int64_t n, lo, hi;
        if (boundary) fine.bface_lattice(f, lat, n, lo, hi);
        else fine.face_lattice(f, lat, n, lo, hi);
        lines[{boundary ? fine.bax[size_t(f)] : fine.fax[size_t(f)], n}].push_back({lo, hi, int32_t(f)});
    }
    for (auto& kv : lines)
        std::sort(kv.second.begin(), kv.second.end(), [](const Seg& a, const Seg& b) { return a.lo < b.lo; });
    ptr.assign(1, 0);
    idx.clear();
    w.clear();
    const int64_t ncoarse = boundary ? int64_t(coarse.bcell.size()) : coarse.nfaces();
    for (int64_t f = 0; f < ncoarse; ++f) {
        int64_t n, lo, hi;
        if (boundary) coarse.bface_lattice(f, lat, n, lo, hi);
        else coarse.face_lattice(f, lat, n, lo, hi);
        auto it = lines.find({boundary ? coarse.bax[size_t(f)] : coarse.fax[size_t(f)], n});
        int64_t covered = 0;
        if (it != lines.end()) {
            const auto& segs = it->second;
            auto p = std::upper_bound(segs.begin(), segs.end(), lo, [](int64_t v, const Seg& s) { return v < s.lo; });
            if (p != segs.begin()) --p;
            for (; p != segs.end() && p->lo < hi; ++p) {
                int64_t ov = std::min(hi, p->hi) - std::max(lo, p->lo);
                if (ov > 0) {
                    idx.push_back(p->f);
                    w.push_back(double(ov) / double(hi - lo));
                    covered += ov;
                }
            }
        }
        if (covered != hi - lo) throw Error(1, "tree hierarchy could not cover a coarse face with fine faces");
        ptr.push_back(int64_t(idx.size()));
    }
}

std::vector<double> restrict_faces(const HostLevel& fine) {
    std::vector<double> out(fine.rptr.size() - 1);
    for (size_t f = 0; f + 1 < fine.rptr.size(); ++f) {
        double v = 0.0;
        for (int64_t k = fine.rptr[f]; k < fine.rptr[f + 1]; ++k) v += fine.rw[size_t(k)] * fine.op.kappa[size_t(fine.ridx[size_t(k)])];
        out[f] = v;
    }
    return out;
}

std::vector<double> restrict_boundary_faces(const HostLevel& fine) {
    std::vector<double> out(fine.brptr.empty() ? 0 : fine.brptr.size() - 1);
    for (size_t f = 0; f < out.size(); ++f) {
        double v = 0.0;
        for (int64_t k = fine.brptr[f]; k < fine.brptr[f + 1]; ++k)
            v += fine.brw[size_t(k)] * fine.op.bkappa[size_t(fine.bridx[size_t(k)])];
        out[f] = v;
    }
    return out;
}

void transfer_weights(HostLevel& lev) {
    std::vector<double> d, rs;
    diag_and_rowsums(lev.op.A, d, rs);
    lev.transfer_inv = d;
    lev.transfer_weight = jacobi_weight(lev.transfer_inv, rs, true, false, false, 0.0);
}

}  // namespace

void finish_level(HostLevel& lev) {
    std::vector<double> rs;
    diag_and_rowsums(lev.op.A, lev.inv_diag, rs);
    lev.weight = jacobi_weight(lev.inv_diag, rs, false, lev.op.singular, true, 1.0);
}

void factor_coarse(Hierarchy& h) {
    const HostLevel& c = h.levels.back();
    const int64_t n = c.op.A.n;
    const int64_t ncomp = c.op.singular ? int64_t(c.op.comp.volume.size()) : 0;
    const int64_t N = n + ncomp;
    if (N > 8192) throw Error(5, "coarsest level exceeds the dense solve limit of 8192 unknowns");
    std::vector<double> M(static_cast<size_t>(N * N), 0.0);
    for (int64_t r = 0; r < n; ++r)
        for (int64_t k = c.op.A.ptr[size_t(r)]; k < c.op.A.ptr[size_t(r + 1)]; ++k)
            M[size_t(r * N + c.op.A.col[size_t(k)])] = c.op.A.val[size_t(k)];
    for (int64_t r = 0; r < n && ncomp; ++r) {
        int32_t s = c.op.comp.slot[size_t(r)];
        if (s < 0) continue;
        M[size_t(r * N + n + s)] = c.op.volumes[size_t(r)];
        M[size_t((n + s) * N + r)] = c.op.volumes[size_t(r)];
    }
    // LU with partial pivoting, then the first n columns of the inverse.
    std::vector<int64_t> piv(static_cast<size_t>(N));
    for (int64_t k = 0; k < N; ++k) {
        int64_t p = k;
        for (int64_t r = k + 1; r < N; ++r)
            if (std::fabs(M[size_t(r * N + k)]) > std::fabs(M[size_t(p * N + k)])) p = r;
        piv[size_t(k)] = p;
        if (M[size_t(p * N + k)] == 0.0) throw Error(1, "coarsest multigrid matrix is singular");
        if (p != k)
            for (int64_t c2 = 0; c2 < N; ++c2) std::swap(M[size_t(k * N + c2)], M[size_t(p * N + c2)]);
        double inv = 1.0 / M[size_t(k * N + k)];
        for (int64_t r = k + 1; r < N; ++r) {
            double l = M[size_t(r * N + k)] * inv;
            M[size_t(r * N + k)] = l;
            if (l != 0.0)
                for (int64_t c2 = k + 1; c2 < N; ++c2) M[size_t(r * N + c2)] -= l * M[size_t(k * N + c2)];
        }
    }
    h.coarse_n = n;
    h.coarse_inverse.assign(static_cast<size_t>(n * n), 0.0);
    std::vector<double> e(static_cast<size_t>(N));
    for (int64_t col = 0; col < n; ++col) {
        std::fill(e.begin(), e.end(), 0.0);
        e[size_t(col)] = 1.0;
        for (int64_t k = 0; k < N; ++k) std::swap(e[size_t(k)], e[size_t(piv[size_t(k)])]);
        for (int64_t r = 0; r < N; ++r) {
            double s = e[size_t(r)];
            for (int64_t k = 0; k < r; ++k) s -= M[size_t(r * N + k)] * e[size_t(k)];
            e[size_t(r)] = s;
        }
        for (int64_t r = N - 1; r >= 0; --r) {
            double s = e[size_t(r)];
            for (int64_t k = r + 1; k < N; ++k) s -= M[size_t(r * N + k)] * e[size_t(k)];
            e[size_t(r)] = s / M[size_t(r * N + r)];
        }
        for (int64_t r = 0; r < n; ++r) h.coarse_inverse[size_t(r * n + col)] = e[size_t(r)];
    }
}

Hierarchy build_hierarchy(LevelOperator fine, const HierarchyOptions& opts) {
    if (opts.coarse_size <= 0) throw Error(1, "coarse_size must be positive");
    if (opts.pre_sweeps < 0 || opts.post_sweeps < 0) throw Error(1, "sweep counts must be nonnegative");
    if (opts.max_levels <= 0) throw Error(1, "max_levels must be positive");
    Hierarchy h;
    h.opts = opts;
    h.levels.emplace_back();
    h.levels.back().op = std::move(fine);
    while (true) {
        HostLevel& cur = h.levels.back();
        Mesh coarse;
        if (!next_coarse(cur.op.mesh, opts, int(h.levels.size()), coarse)) break;
        cur.owner = owners(cur.op.mesh, coarse);
        transfer_weights(cur);
        face_restriction(coarse, cur.op.mesh, cur.rptr, cur.ridx, cur.rw);
        std::vector<double> kc = restrict_faces(cur);
        HostLevel next;
        // open sides keep their conductance on every level, with the boundary
        // coefficients restricted like the interior ones
        // (geometric_preconditioner.jl:256-300)
        for (int s = 0; s < 4; ++s) next.op.open[s] = cur.op.open[s];
        if (cur.op.any_open()) {
            face_restriction(coarse, cur.op.mesh, cur.brptr, cur.bridx, cur.brw, true);
            next.op.bkappa = restrict_boundary_faces(cur);
        }
        next.op.mesh = std::move(coarse);
        next.op.metric = assemble_metric(next.op.mesh);
        next.op.kappa = std::move(kc);
        assemble_operator(next.op);
        h.levels.push_back(std::move(next));
    }
    for (auto& lev : h.levels) finish_level(lev);
    factor_coarse(h);
    return h;
}

void refresh_hierarchy(Hierarchy& h, const std::vector<double>& kappa) {
    h.levels[0].op.kappa = kappa;
    assemble_operator(h.levels[0].op);
    for (size_t l = 1; l < h.levels.size(); ++l) {
        h.levels[l].op.kappa = restrict_faces(h.levels[l - 1]);
        if (h.levels[l].op.any_open()) h.levels[l].op.bkappa = restrict_boundary_faces(h.levels[l - 1]);
        assemble_operator(h.levels[l].op);
    }
    for (size_t l = 0; l + 1 < h.levels.size(); ++l) transfer_weights(h.levels[l]);
    for (auto& lev : h.levels) finish_level(lev);
    factor_coarse(h);
}

}  // namespace tpa
