// Block-structured (stencil + exception rows) form of an assembled level.
//
// A level's matrix is the rediscretised operator of its composite block mesh
// (src/operators/elliptic.jl:157-257 in ronaldremmerswaal/TwoPhaseAMR.jl).  On
// every row whose couplings are exactly the four lattice neighbours of the
// same size (inside the block, or in the same-size neighbour block across a
// block edge, periodic seams included) the row is a 5-point stencil with the
// coupling -a_ij stored once per face (east face in cx, north face in cy) and
// a_ii equal to the sum of its four face coefficients.  Every other row (cells
// next to a coarse-fine block edge, where the non-diagonal vertex-patch metric
// of gradient.jl:194-232 couples more cells) keeps its assembled CSR row as an
// exception.  The tentative transfer of the tree hierarchy maps every fine
// block onto a quadrant of one coarse block (scale 2: four sibling blocks or
// four roots merged) or onto a whole coarse block (scale 1: a block kept by
// the pruning), tree_coarsening.jl:30-82, 228-252.
#include <algorithm>
#include <cmath>

#include "structure.hpp"

namespace tpa {

namespace {

bool near(double a, double b, double rel) { return std::fabs(a - b) <= rel * std::max(std::fabs(a), std::fabs(b)); }

}  // namespace

StructLevel build_struct(const HostLevel& lev, const Mesh* coarse_mesh) {
    const Mesh& m = lev.op.mesh;
    const Csr& A = lev.op.A;
    StructLevel s;
    s.nx = m.bs[0];
    s.ny = m.bs[1];
    const int nx = s.nx, ny = s.ny, cpb = nx * ny;
    const int64_t nb = m.nblocks();
    s.nblocks = nb;
    s.nbr.assign(size_t(4 * nb), -1);
    for (int64_t b = 0; b < nb; ++b) {
        uint64_t k = m.keys[size_t(b)];
        int lev_ = key_level(k);
        int64_t i = key_i(k), j = key_j(k);
        int64_t nxl = int64_t(m.forest.layout[0]) << lev_, nyl = int64_t(m.forest.layout[1]) << lev_;
        const int64_t di[4] = {-1, 1, 0, 0}, dj[4] = {0, 0, -1, 1};
        for (int d = 0; d < 4; ++d) {
            int64_t ni = i + di[d], nj = j + dj[d];
            if (m.periodic[0]) ni = ((ni % nxl) + nxl) % nxl;
            else if (ni < 0 || ni >= nxl) continue;
            if (m.periodic[1]) nj = ((nj % nyl) + nyl) % nyl;
            else if (nj < 0 || nj >= nyl) continue;
            auto it = m.index.find(pack_key(lev_, ni, nj));
            if (it != m.index.end()) s.nbr[size_t(4 * b + d)] = it->second;
        }
    }
    const int64_t n = m.ncells();
    s.cx.assign(size_t(n), 0.0);
    s.cy.assign(size_t(n), 0.0);
    s.ex.assign(size_t(n), -1);
    s.ex_ptr.assign(1, 0);
    // structured neighbour of cell c in direction d (0 W, 1 E, 2 S, 3 N), or -1
    auto neighbour = [&](int64_t c, int d) -> int64_t {
        int64_t b = c / cpb, r = c % cpb;
        int i = int(r % nx), j = int(r / nx);
        int ni = i + (d == 0 ? -1 : d == 1 ? 1 : 0), nj = j + (d == 2 ? -1 : d == 3 ? 1 : 0);
        if (ni >= 0 && ni < nx && nj >= 0 && nj < ny) return b * cpb + nj * nx + ni;
        int32_t q = s.nbr[size_t(4 * b + d)];
        if (q < 0) return -1;
        ni = (ni + nx) % nx;
        nj = (nj + ny) % ny;
        return int64_t(q) * cpb + nj * nx + ni;
    };
    int64_t exceptions = 0;
    bool first_coef = true;
    double c0 = 0.0;
    s.const_coef = true;
    std::vector<char> regular(size_t(n), 0);
    for (int64_t c = 0; c < n; ++c) {
        int64_t nbc[4];
        for (int d = 0; d < 4; ++d) nbc[d] = neighbour(c, d);
        // row must hold exactly {c} and the existing structured neighbours
        bool ok = true;
        double coef[4] = {0, 0, 0, 0}, diag = 0;
        int found = 0, nonself = 0;
        for (int64_t k = A.ptr[size_t(c)]; k < A.ptr[size_t(c + 1)] && ok; ++k) {
            int32_t col = A.col[size_t(k)];
            double v = A.val[size_t(k)];
            if (col == c) {
                diag = v;
                continue;
            }
            ++nonself;
            int match = -1;
            for (int d = 0; d < 4; ++d)
                if (nbc[d] == col && match < 0) match = d;
            if (match < 0) {
                ok = v == 0.0;  // an explicit zero outside the stencil is harmless
                continue;
            }
            // a neighbour may appear once per direction; two directions to one cell
            // (a two-cell periodic axis) makes the row irregular
            for (int d = match + 1; d < 4; ++d)
                if (nbc[d] == col) ok = false;
            coef[match] = -v;
            ++found;
        }
        // a missing in-mesh neighbour would mean a zero coupling, which is fine
        double sum = coef[0] + coef[1] + coef[2] + coef[3];
        if (ok && !near(diag, sum, 1e-12) && !(diag == 0 && sum == 0)) ok = false;
        (void)found;
        (void)nonself;
        if (ok) {
            regular[size_t(c)] = 1;
            // store the east and north coefficients on this cell; the west and
            // south ones are the east / north coefficients of the neighbours
            if (nbc[1] >= 0) s.cx[size_t(c)] = coef[1];
            if (nbc[3] >= 0) s.cy[size_t(c)] = coef[3];
        } else {
            s.ex[size_t(c)] = int32_t(exceptions++);
            for (int64_t k = A.ptr[size_t(c)]; k < A.ptr[size_t(c + 1)]; ++k) {
                s.ex_col.push_back(A.col[size_t(k)]);
                s.ex_val.push_back(A.val[size_t(k)]);
            }
            s.ex_ptr.push_back(int64_t(s.ex_col.size()));
        }
    }
    // West / south coefficients of a regular cell come from its neighbours'
    // east / north entries: the neighbour must have stored them.  A regular cell
    // whose west neighbour is an exception row still needs that coefficient.
    for (int64_t c = 0; c < n; ++c) {
        if (!regular[size_t(c)]) continue;
        for (int d : {0, 2}) {
            int64_t q = neighbour(c, d);
            if (q < 0) continue;
            double v = 0;
            for (int64_t k = A.ptr[size_t(c)]; k < A.ptr[size_t(c + 1)]; ++k)
                if (A.col[size_t(k)] == q) v = -A.val[size_t(k)];
            if (d == 0) s.cx[size_t(q)] = v;
            else s.cy[size_t(q)] = v;
        }
    }
    for (int64_t c = 0; c < n; ++c) {
        if (!regular[size_t(c)]) continue;
        for (int d = 0; d < 4; ++d) {
            int64_t q = neighbour(c, d);
            if (q < 0) continue;
            double v = d == 0 ? s.cx[size_t(q)] : d == 1 ? s.cx[size_t(c)] : d == 2 ? s.cy[size_t(q)] : s.cy[size_t(c)];
            if (first_coef) {
                c0 = v;
                first_coef = false;
            } else if (!near(v, c0, 1e-13)) {
                s.const_coef = false;
            }
        }
    }
    s.c0 = c0;
    s.nex = exceptions;
    s.dinv = lev.inv_diag;
    // constant diagonal: every regular and exception row has the same D^-1
    s.const_diag = true;
    for (int64_t c = 1; c < n && s.const_diag; ++c)
        if (!near(s.dinv[size_t(c)], s.dinv[0], 1e-13)) s.const_diag = false;
    s.tinv_same = true;
    for (size_t c = 0; c < lev.transfer_inv.size() && s.tinv_same; ++c)
        if (lev.transfer_inv[c] != lev.inv_diag[c]) s.tinv_same = false;
    // block map of the tentative transfer
    s.has_map = false;
    if (coarse_mesh && !lev.owner.empty()) {
        s.map.assign(size_t(4 * nb), 0);
        bool good = true;
        for (int64_t b = 0; b < nb && good; ++b) {
            int64_t o00 = lev.owner[size_t(b * cpb)];
            int64_t o11 = lev.owner[size_t(b * cpb + nx + 1)];
            int64_t cb = o00 / cpb, r0 = o00 % cpb;
            int scale = (o11 == o00) ? 2 : 1;
            int ox = int(r0 % nx), oy = int(r0 / nx);
            for (int j = 0; j < ny && good; ++j)
                for (int i = 0; i < nx && good; ++i) {
                    int64_t expect = cb * cpb + (oy + j / scale) * nx + (ox + i / scale);
                    if (lev.owner[size_t(b * cpb + j * nx + i)] != expect) good = false;
                }
            s.map[size_t(4 * b)] = int32_t(cb);
            s.map[size_t(4 * b + 1)] = ox;
            s.map[size_t(4 * b + 2)] = oy;
            s.map[size_t(4 * b + 3)] = scale;
        }
        s.has_map = good;
    }
    return s;
}

}  // namespace tpa
