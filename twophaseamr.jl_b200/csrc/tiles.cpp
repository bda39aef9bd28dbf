// Haloed block tiles of a CSR level (see tiles.hpp).
#include "tiles.hpp"

#include <algorithm>

namespace tpa {

TileLevelHost build_tiles(const Csr& A, int64_t nblocks, int64_t cpb, const std::vector<int32_t>& owner, int64_t nc,
                          int max_cells) {
    TileLevelHost T;
    const int64_t n = A.n;
    if (nblocks <= 0 || cpb <= 0 || nblocks * cpb != n || int64_t(owner.size()) != n || nc <= 0 ||
        cpb > max_cells)
        return T;
    // children of every coarse cell, in increasing fine-cell order (the order of
    // the device child lists)
    std::vector<int64_t> cptr(size_t(nc + 1), 0);
    for (int32_t o : owner) {
        if (o < 0 || o >= nc) return T;
        cptr[size_t(o) + 1]++;
    }
    for (int64_t J = 0; J < nc; ++J) {
        if (cptr[size_t(J) + 1] < 1 || cptr[size_t(J) + 1] > 4) return T;
        cptr[size_t(J) + 1] += cptr[size_t(J)];
    }
    std::vector<int32_t> kids(static_cast<size_t>(n));
    {
        std::vector<int64_t> next(cptr.begin(), cptr.end() - 1);
        for (int64_t i = 0; i < n; ++i) kids[size_t(next[size_t(owner[size_t(i)])]++)] = int32_t(i);
    }
    std::vector<int32_t> loc(size_t(n), -1);
    std::vector<char> seen(size_t(nc), 0);
    T.ntiles = int(nblocks);
    T.cell_off.push_back(0);
    T.lrp_off.push_back(0);
    T.ent_off.push_back(0);
    T.co_off.push_back(0);
    std::vector<int32_t> cells;
    for (int64_t t = 0; t < nblocks; ++t) {
        cells.clear();
        for (int64_t k = 0; k < cpb; ++k) {
            const int32_t g = int32_t(t * cpb + k);
            loc[size_t(g)] = int32_t(k);
            cells.push_back(g);
        }
        int ring[4] = {int(cpb), 0, 0, 0};
        size_t begin = 0, end = cells.size();
        for (int r = 1; r <= 3; ++r) {
            for (size_t k = begin; k < end; ++k) {
                const int32_t g = cells[k];
                for (int64_t e = A.ptr[size_t(g)]; e < A.ptr[size_t(g) + 1]; ++e) {
                    const int32_t j = A.col[size_t(e)];
                    if (loc[size_t(j)] < 0) {
                        loc[size_t(j)] = int32_t(cells.size());
                        cells.push_back(j);
                    }
                }
            }
            begin = end;
            end = cells.size();
            ring[r] = int(end);
        }
        bool fits = ring[3] <= max_cells;
        // local rows of rings <= 2: every column is a local cell by construction
        const int n2 = ring[2];
        const size_t e_begin = T.pos.size();
        for (int k = 0; k < n2 && fits; ++k) {
            const int32_t g = cells[size_t(k)];
            T.lrp.push_back(int32_t(T.pos.size() - e_begin));
            for (int64_t e = A.ptr[size_t(g)]; e < A.ptr[size_t(g) + 1]; ++e) {
                const int32_t lc = loc[size_t(A.col[size_t(e)])];
                if (lc < 0 || lc >= ring[3]) fits = false;
                T.pos.push_back(int32_t(e));
                T.lcol.push_back(int16_t(lc));
            }
        }
        T.lrp.push_back(int32_t(T.pos.size() - e_begin));
        const int64_t ne = int64_t(T.pos.size() - e_begin);
        if (ne > 32767) fits = false;
        // coarse cells of the block, in order of their first child
        int nco = 0;
        for (int64_t k = 0; k < cpb && fits; ++k) {
            const int32_t J = owner[size_t(t * cpb + k)];
            if (seen[size_t(J)]) continue;
            seen[size_t(J)] = 1;
            T.co.push_back(J);
            ++nco;
            int16_t q4[4] = {-1, -1, -1, -1};
            for (int64_t c = cptr[size_t(J)], q = 0; c < cptr[size_t(J) + 1]; ++c, ++q) {
                const int32_t lc = loc[size_t(kids[size_t(c)])];
                if (lc < 0 || lc >= int32_t(cpb)) fits = false;  // a child outside the block
                q4[q] = int16_t(lc);
            }
            for (int q = 0; q < 4; ++q) T.ch.push_back(q4[q]);
        }
        for (int32_t g : cells) loc[size_t(g)] = -1;
        if (!fits) return TileLevelHost();
        T.cell.insert(T.cell.end(), cells.begin(), cells.end());
        for (int32_t g : cells) T.own.push_back(owner[size_t(g)]);
        for (int r = 0; r < 4; ++r) T.ring.push_back(ring[r]);
        T.cell_off.push_back(int32_t(T.cell.size()));
        T.lrp_off.push_back(int32_t(T.lrp.size()));
        T.ent_off.push_back(int32_t(T.pos.size()));
        T.co_off.push_back(int32_t(T.co.size()));
        T.n3max = std::max(T.n3max, ring[3]);
        T.n2max = std::max(T.n2max, ring[2]);
        T.n1max = std::max(T.n1max, ring[1]);
        T.emax = std::max<int>(T.emax, int(ne));
        T.comax = std::max(T.comax, nco);
    }
    // every coarse cell belongs to exactly one tile
    if (int64_t(T.co.size()) != nc) return TileLevelHost();
    if (T.cell.size() > size_t(INT32_MAX) || T.pos.size() > size_t(INT32_MAX)) return TileLevelHost();
    T.ok = true;
    return T;
}

}  // namespace tpa
