// Block forest, leaf order and face schedules.
//
// Reproduces (ronaldremmerswaal/TwoPhaseAMR.jl):
//   src/mesh/topology/mesh.jl:673-714   `_balance!`: minimal 2:1 grading across
//                                       faces and corners, periodic seams included
//   src/mesh/topology/mesh.jl:759-773   `_leaf_blocks`: blocks sorted by (level, j, i)
//   src/mesh/topology/mesh.jl:787-937   `_lattice_sides`/`_match_sides!`: faces on the
//                                       finest active lattice, axis-major, then by line,
//                                       then by tangential position; boundary faces
//   src/mesh/topology/mesh.jl:450-474   lattice bounds of cells and faces
#include <algorithm>
#include <numeric>

#include "host.hpp"

namespace tpa {

void Forest::node_box(uint64_t key, double o[2], double e[2]) const {
    int level = key_level(key);
    int64_t i = key_i(key), j = key_j(key);
    if (level == 0) {
        o[0] = origin[0] + double(i) * root_extent[0];
        o[1] = origin[1] + double(j) * root_extent[1];
        e[0] = root_extent[0];
        e[1] = root_extent[1];
        return;
    }
    double po[2], pe[2];
    node_box(pack_key(level - 1, i >> 1, j >> 1), po, pe);
    e[0] = pe[0] / 2;
    e[1] = pe[1] / 2;
    o[0] = (i & 1) ? po[0] + e[0] : po[0];
    o[1] = (j & 1) ? po[1] + e[1] : po[1];
}

void Forest::split(uint64_t key) {
    leaves.erase(key);
    internal.insert(key);
    int level = key_level(key);
    int64_t i = key_i(key), j = key_j(key);
    for (int cj = 0; cj < 2; ++cj)
        for (int ci = 0; ci < 2; ++ci) leaves.insert(pack_key(level + 1, 2 * i + ci, 2 * j + cj));
}

bool Forest::leaf_at(int level, int64_t i, int64_t j, uint64_t& out) const {
    for (int l = 0; l <= level; ++l) {
        uint64_t k = pack_key(l, i >> (level - l), j >> (level - l));
        if (leaves.count(k)) {
            out = k;
            return true;
        }
        if (!internal.count(k)) return false;
    }
    return false;
}

void Forest::balance(const bool periodic[2]) {
    bool changed = true;
    std::vector<uint64_t> work;
    while (changed) {
        changed = false;
        work.assign(leaves.begin(), leaves.end());
        std::sort(work.begin(), work.end());
        for (uint64_t leaf : work) {
            if (!leaves.count(leaf)) continue;
            int level = key_level(leaf);
            if (level < 2) continue;
            int64_t i = key_i(leaf), j = key_j(leaf);
            int64_t nxl = int64_t(layout[0]) << level, nyl = int64_t(layout[1]) << level;
            for (int dj = -1; dj <= 1; ++dj)
                for (int di = -1; di <= 1; ++di) {
                    if (!di && !dj) continue;
                    int64_t ni = i + di, nj = j + dj;
                    if (periodic[0]) ni = ((ni % nxl) + nxl) % nxl;
                    else if (ni < 0 || ni >= nxl) continue;
                    if (periodic[1]) nj = ((nj % nyl) + nyl) % nyl;
                    else if (nj < 0 || nj >= nyl) continue;
                    uint64_t cover;
                    if (leaf_at(level, ni, nj, cover) && key_level(cover) + 1 < level) {
                        split(cover);
                        changed = true;
                    }
                }
        }
    }
}

void Mesh::cell_lattice(int64_t cell, const int64_t lat[2], int64_t low[2], int64_t sc[2]) const {
    int64_t cpb = cells_per_block();
    int64_t b = cell / cpb, r = cell % cpb;
    int64_t i = r % bs[0], j = r / bs[0];
    uint64_t k = keys[size_t(b)];
    int lev = key_level(k);
    sc[0] = lat[0] / (int64_t(base[0]) << lev);
    sc[1] = lat[1] / (int64_t(base[1]) << lev);
    low[0] = (key_i(k) * bs[0] + i) * sc[0];
    low[1] = (key_j(k) * bs[1] + j) * sc[1];
}

void Mesh::face_lattice(int64_t f, const int64_t lat[2], int64_t& normal, int64_t& lo, int64_t& hi) const {
    int64_t ml[2], ms[2], pl[2], ps[2];
    cell_lattice(fm[size_t(f)], lat, ml, ms);
    cell_lattice(fp[size_t(f)], lat, pl, ps);
    int a = fax[size_t(f)] - 1, t = 1 - a;
    normal = ml[a] + ms[a];
    if (periodic[a]) normal = ((normal % lat[a]) + lat[a]) % lat[a];
    lo = std::max(ml[t], pl[t]);
    hi = std::min(ml[t] + ms[t], pl[t] + ps[t]);
}

void Mesh::bface_lattice(int64_t b, const int64_t lat[2], int64_t& normal, int64_t& lo, int64_t& hi) const {
    int64_t low[2], sc[2];
    cell_lattice(bcell[size_t(b)], lat, low, sc);
    const int a = bax[size_t(b)] - 1, t = 1 - a;
    normal = low[a] + (bside[size_t(b)] > 0 ? sc[a] : 0);
    lo = low[t];
    hi = low[t] + sc[t];
}

std::vector<double> Mesh::cell_volumes() const {
    std::vector<double> v(static_cast<size_t>(ncells()));
    int64_t cpb = cells_per_block();
    for (int64_t b = 0; b < nblocks(); ++b)
        std::fill(v.begin() + b * cpb, v.begin() + (b + 1) * cpb, bvol[size_t(b)]);
    return v;
}

namespace {

struct Side {
    int64_t lo, hi;
    int32_t cell;
};

// `_lattice_sides` + `_match_sides!` for one axis (0-based axis `a`).
void match_axis(Mesh& m, int a, const int64_t lat[2]) {
    const int nx = m.bs[0], ny = m.bs[1];
    const int t = 1 - a;
    const int64_t lines = lat[a];
    const int64_t nb = m.nblocks(), cpb = m.cells_per_block();
    std::vector<int64_t> lower_count(static_cast<size_t>(lines + 2), 0), upper_count(static_cast<size_t>(lines + 2), 0);
    auto side_of = [&](int64_t cell, int64_t& low, int64_t& high, int64_t& tlo, int64_t& thi) {
        int64_t b = cell / cpb, r = cell % cpb;
        uint64_t k = m.keys[size_t(b)];
        int64_t scale = int64_t(1) << (m.active - key_level(k));
        int64_t xlo = key_i(k) * nx * scale + (r % nx) * scale;
        int64_t ylo = key_j(k) * ny * scale + (r / nx) * scale;
        if (a == 0) { low = xlo; high = xlo + scale; tlo = ylo; thi = ylo + scale; }
        else        { low = ylo; high = ylo + scale; tlo = xlo; thi = xlo + scale; }
    };
    auto canon = [&](int64_t c) { return m.periodic[a] ? ((c % lines) + lines) % lines : c; };
    const int64_t nc = nb * cpb;
    for (int64_t c = 0; c < nc; ++c) {
        int64_t low, high, tlo, thi;
        side_of(c, low, high, tlo, thi);
        lower_count[size_t(canon(high) + 1)]++;
        upper_count[size_t(canon(low) + 1)]++;
    }
    for (int64_t l = 0; l <= lines; ++l) {
        lower_count[size_t(l + 1)] += lower_count[size_t(l)];
        upper_count[size_t(l + 1)] += upper_count[size_t(l)];
    }
    std::vector<Side> lower(static_cast<size_t>(nc)), upper(static_cast<size_t>(nc));
    std::vector<int64_t> ln(lower_count.begin(), lower_count.end() - 1), un(upper_count.begin(), upper_count.end() - 1);
    for (int64_t c = 0; c < nc; ++c) {
        int64_t low, high, tlo, thi;
        side_of(c, low, high, tlo, thi);
        Side s{tlo, thi, int32_t(c)};
        lower[size_t(ln[size_t(canon(high))]++)] = s;
        upper[size_t(un[size_t(canon(low))]++)] = s;
    }
    auto by_lo = [](const Side& x, const Side& y) { return x.lo < y.lo; };
    const double normal_scale = m.extent[a] / double(lat[a]);
    const double tangent_scale = m.extent[t] / double(lat[t]);
    (void)normal_scale;
    for (int64_t line = 0; line <= lines; ++line) {
        int64_t li = lower_count[size_t(line)], lstop = lower_count[size_t(line + 1)];
        int64_t ui = upper_count[size_t(line)], ustop = upper_count[size_t(line + 1)];
        std::sort(lower.begin() + li, lower.begin() + lstop, by_lo);
        std::sort(upper.begin() + ui, upper.begin() + ustop, by_lo);
        while (li < lstop && ui < ustop) {
            const Side& L = lower[size_t(li)];
            const Side& U = upper[size_t(ui)];
            int64_t lo = std::max(L.lo, U.lo), hi = std::min(L.hi, U.hi);
            if (lo < hi) {
                m.fm.push_back(L.cell);
                m.fp.push_back(U.cell);
                m.fax.push_back(int8_t(a + 1));
                m.farea.push_back(double(hi - lo) * tangent_scale);
            }
            int64_t lh = L.hi, uh = U.hi;
            if (lh <= uh) ++li;
            if (uh <= lh) ++ui;
        }
        for (; li < lstop; ++li) {
            const Side& s = lower[size_t(li)];
            m.bcell.push_back(s.cell); m.bax.push_back(int8_t(a + 1)); m.bside.push_back(1);
            m.barea.push_back(double(s.hi - s.lo) * m.extent[t] / double(lat[t]));
        }
        for (; ui < ustop; ++ui) {
            const Side& s = upper[size_t(ui)];
            m.bcell.push_back(s.cell); m.bax.push_back(int8_t(a + 1)); m.bside.push_back(-1);
            m.barea.push_back(double(s.hi - s.lo) * m.extent[t] / double(lat[t]));
        }
    }
}

}  // namespace

Mesh mesh_from_forest(Forest forest, const int base[2], const int bs[2], const bool periodic[2]) {
    Mesh m;
    for (int a = 0; a < 2; ++a) {
        m.base[a] = base[a];
        m.bs[a] = bs[a];
        m.periodic[a] = periodic[a];
        m.origin[a] = forest.origin[a];
        m.extent[a] = forest.extent[a];
    }
    m.keys.assign(forest.leaves.begin(), forest.leaves.end());
    std::sort(m.keys.begin(), m.keys.end(), [](uint64_t x, uint64_t y) {
        int lx = key_level(x), ly = key_level(y);
        if (lx != ly) return lx < ly;
        if (key_j(x) != key_j(y)) return key_j(x) < key_j(y);
        return key_i(x) < key_i(y);
    });
    size_t nb = m.keys.size();
    m.bsx.resize(nb); m.bsy.resize(nb); m.bvol.resize(nb); m.box.resize(nb); m.boy.resize(nb);
    m.active = 0;
    for (size_t b = 0; b < nb; ++b) {
        double o[2], e[2];
        forest.node_box(m.keys[b], o, e);
        m.box[b] = o[0]; m.boy[b] = o[1];
        m.bsx[b] = e[0] / bs[0];
        m.bsy[b] = e[1] / bs[1];
        m.bvol[b] = m.bsx[b] * m.bsy[b];
        m.index[m.keys[b]] = int32_t(b);
        m.active = std::max(m.active, key_level(m.keys[b]));
    }
    m.forest = std::move(forest);
    int64_t lat[2];
    m.lattice(m.active, lat);
    match_axis(m, 0, lat);
    match_axis(m, 1, lat);
    return m;
}

Mesh build_mesh(const int base[2], const int bs[2], const bool periodic[2], const double origin[2],
                const double extent[2], const std::vector<uint64_t>& leaves) {
    for (int a = 0; a < 2; ++a) {
        if (bs[a] < 2 || bs[a] % 2) throw Error(1, "block dimensions must be even and at least two");
        if (base[a] < bs[a] || base[a] % bs[a])
            throw Error(1, "base mesh dimensions must be integer multiples of block dimensions");
        if (!(extent[a] > 0)) throw Error(1, "domain extents must be positive");
    }
    Forest f;
    for (int a = 0; a < 2; ++a) {
        f.layout[a] = base[a] / bs[a];
        f.origin[a] = origin[a];
        f.extent[a] = extent[a];
        f.root_extent[a] = extent[a] / f.layout[a];
    }
    for (uint64_t k : leaves) {
        int lev = key_level(k);
        int64_t i = key_i(k), j = key_j(k);
        if (lev > 28 || i >= (int64_t(f.layout[0]) << lev) || j >= (int64_t(f.layout[1]) << lev))
            throw Error(1, "leaf key outside the root layout");
        f.leaves.insert(k);
        for (int l = 0; l < lev; ++l) f.internal.insert(pack_key(l, i >> (lev - l), j >> (lev - l)));
    }
    for (uint64_t k : f.internal) f.leaves.erase(k);
    // every root must be covered
    for (int j = 0; j < f.layout[1]; ++j)
        for (int i = 0; i < f.layout[0]; ++i) {
            uint64_t k = pack_key(0, i, j);
            if (!f.leaves.count(k) && !f.internal.count(k)) throw Error(1, "leaf set does not cover every root");
        }
    // every internal node must have its four children present
    for (uint64_t k : f.internal) {
        int lev = key_level(k);
        for (int cj = 0; cj < 2; ++cj)
            for (int ci = 0; ci < 2; ++ci) {
                uint64_t c = pack_key(lev + 1, 2 * key_i(k) + ci, 2 * key_j(k) + cj);
                if (!f.leaves.count(c) && !f.internal.count(c)) throw Error(1, "leaf set is not a complete quadtree");
            }
    }
    f.balance(periodic);
    return mesh_from_forest(std::move(f), base, bs, periodic);
}

}  // namespace tpa
