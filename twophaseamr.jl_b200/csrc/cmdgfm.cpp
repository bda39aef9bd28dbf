// Host set-up of the CMDGFM two-block solve (cmdgfm.hpp).  Compiled by the
// host compiler without contraction of multiply-adds, so the factor has the
// bits of the oracle's restatement (oracle/cmdgfm.py), which sums in the same
// orders.
#include "cmdgfm.hpp"

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <string>
#include <utility>

#include "host.hpp"

namespace tpa {

namespace {

// A dense accumulator over [0, n) that remembers which entries it touched.
struct Accumulator {
    std::vector<double> v;
    std::vector<char> mark;
    std::vector<int32_t> touched;
    explicit Accumulator(int64_t n) : v(size_t(n), 0.0), mark(size_t(n), 0) {}
    // value of entry j (0.0 when untouched): the first touch stores 0.0 first
    double& at(int32_t j) {
        if (!mark[size_t(j)]) {
            mark[size_t(j)] = 1;
            v[size_t(j)] = 0.0;
            touched.push_back(j);
        }
        return v[size_t(j)];
    }
    void sort() { std::sort(touched.begin(), touched.end()); }
    void clear() {
        for (int32_t j : touched) mark[size_t(j)] = 0;
        touched.clear();
    }
};

void push_row(CsrRows& m, const std::vector<std::pair<int32_t, double>>& row) {
    for (const auto& e : row) {
        m.col.push_back(e.first);
        m.val.push_back(e.second);
    }
    m.ptr.push_back(int64_t(m.col.size()));
}

}  // namespace

CsrRows cmdgfm_schur(const CsrRows& m, int64_t np) {
    const int64_t n = m.n, nx = n - np;
    std::vector<double> diag(static_cast<size_t>(np), 0.0);
    std::vector<char> has(static_cast<size_t>(np), 0);
    for (int64_t c = 0; c < np; ++c)
        for (int64_t k = m.ptr[size_t(c)]; k < m.ptr[size_t(c) + 1]; ++k)
            if (m.col[size_t(k)] == c) {
                diag[size_t(c)] = m.val[size_t(k)];
                has[size_t(c)] = 1;
            }
    CsrRows s;
    s.n = nx;
    s.ptr.assign(1, 0);
    Accumulator acc(std::max<int64_t>(nx, 1));
    for (int64_t f = 0; f < nx; ++f) {
        const int64_t r = np + f;
        for (int64_t k = m.ptr[size_t(r)]; k < m.ptr[size_t(r) + 1]; ++k) {
            const int32_t j = m.col[size_t(k)];
            if (j >= np) acc.at(int32_t(j - np)) += m.val[size_t(k)];
        }
        for (int64_t k = m.ptr[size_t(r)]; k < m.ptr[size_t(r) + 1]; ++k) {
            const int32_t c = m.col[size_t(k)];
            if (c >= np) continue;
            if (!has[size_t(c)] || diag[size_t(c)] == 0.0)
                throw Error(1, "the pressure block has a zero diagonal in row " + std::to_string(c));
            const double cval = m.val[size_t(k)];
            for (int64_t kk = m.ptr[size_t(c)]; kk < m.ptr[size_t(c) + 1]; ++kk) {
                const int32_t j = m.col[size_t(kk)];
                if (j < np) continue;
                acc.at(int32_t(j - np)) += -(cval * (m.val[size_t(kk)] / diag[size_t(c)]));
            }
        }
        acc.sort();
        for (int32_t g : acc.touched) {
            s.col.push_back(g);
            s.val.push_back(acc.v[size_t(g)]);
        }
        s.ptr.push_back(int64_t(s.col.size()));
        acc.clear();
    }
    return s;
}

void crout_ilu(const CsrRows& a, double tau, CsrRows& lower, CsrRows& upper, std::vector<double>& pivot) {
    const int64_t n = a.n;
    // column view of A: rows in increasing order per column
    std::vector<std::vector<std::pair<int32_t, double>>> acol(static_cast<size_t>(n));
    for (int64_t r = 0; r < n; ++r)
        for (int64_t k = a.ptr[size_t(r)]; k < a.ptr[size_t(r) + 1]; ++k)
            acol[size_t(a.col[size_t(k)])].emplace_back(int32_t(r), a.val[size_t(k)]);
    using Entries = std::vector<std::pair<int32_t, double>>;
    const size_t nn = static_cast<size_t>(n);
    std::vector<Entries> urow(nn), ucol(nn), lrow(nn), lcol(nn);
    Accumulator u(std::max<int64_t>(n, 1)), l(std::max<int64_t>(n, 1));
    pivot.assign(size_t(n), 0.0);
    for (int64_t k = 0; k < n; ++k) {
        for (int64_t e = a.ptr[size_t(k)]; e < a.ptr[size_t(k) + 1]; ++e)
            if (a.col[size_t(e)] >= k) u.at(a.col[size_t(e)]) = a.val[size_t(e)];
        for (const auto& li : lrow[size_t(k)]) {  // i increasing
            const double lki = li.second;
            for (const auto& uj : urow[size_t(li.first)])
                if (uj.first >= k) {
                    double& x = u.at(uj.first);
                    x = x - lki * uj.second;
                }
        }
        for (const auto& ar : acol[size_t(k)])
            if (ar.first > k) l.at(ar.first) = ar.second;
        for (const auto& ui : ucol[size_t(k)]) {  // i increasing
            const double uik = ui.second;
            for (const auto& lr : lcol[size_t(ui.first)])
                if (lr.first > k) {
                    double& x = l.at(lr.first);
                    x = x - uik * lr.second;
                }
        }
        const double d = u.mark[size_t(k)] ? u.v[size_t(k)] : 0.0;
        if (d == 0.0) throw Error(1, "zero pivot in the incomplete LU of the jump block, row " + std::to_string(k));
        pivot[size_t(k)] = d;
        u.sort();
        for (int32_t j : u.touched) {
            const double x = u.v[size_t(j)];
            if (j == k) continue;
            if (std::fabs(x) >= tau) {
                urow[size_t(k)].emplace_back(j, x);
                ucol[size_t(j)].emplace_back(int32_t(k), x);
            }
        }
        const double inv = 1.0 / d;
        l.sort();
        for (int32_t r : l.touched) {
            const double x = l.v[size_t(r)];
            if (std::fabs(x) >= tau) {
                const double y = x * inv;
                lcol[size_t(k)].emplace_back(r, y);
                lrow[size_t(r)].emplace_back(int32_t(k), y);
            }
        }
        u.clear();
        l.clear();
    }
    lower = CsrRows();
    upper = CsrRows();
    lower.n = upper.n = n;
    lower.ptr.assign(1, 0);
    upper.ptr.assign(1, 0);
    for (int64_t r = 0; r < n; ++r) {
        push_row(lower, lrow[size_t(r)]);
        push_row(upper, urow[size_t(r)]);
    }
}

LevelSchedule forward_levels(const CsrRows& lower) {
    const int64_t n = lower.n;
    std::vector<int32_t> level(static_cast<size_t>(n), 0);
    int32_t depth = 0;
    for (int64_t k = 0; k < n; ++k) {
        int32_t lv = 0;
        for (int64_t e = lower.ptr[size_t(k)]; e < lower.ptr[size_t(k) + 1]; ++e)
            lv = std::max(lv, level[size_t(lower.col[size_t(e)])] + 1);
        level[size_t(k)] = lv;
        depth = std::max(depth, lv + 1);
    }
    LevelSchedule s;
    s.level_ptr.assign(size_t(depth) + 1, 0);
    for (int64_t k = 0; k < n; ++k) ++s.level_ptr[size_t(level[size_t(k)]) + 1];
    for (int32_t d = 0; d < depth; ++d) s.level_ptr[size_t(d) + 1] += s.level_ptr[size_t(d)];
    s.rows.assign(size_t(n), 0);
    std::vector<int32_t> cur(s.level_ptr.begin(), s.level_ptr.end() - 1);
    for (int64_t k = 0; k < n; ++k) s.rows[size_t(cur[size_t(level[size_t(k)])]++)] = int32_t(k);
    return s;
}

LevelSchedule backward_levels(const CsrRows& upper) {
    const int64_t n = upper.n;
    std::vector<int32_t> level(static_cast<size_t>(n), 0);
    int32_t depth = 0;
    for (int64_t k = n - 1; k >= 0; --k) {
        int32_t lv = 0;
        for (int64_t e = upper.ptr[size_t(k)]; e < upper.ptr[size_t(k) + 1]; ++e)
            lv = std::max(lv, level[size_t(upper.col[size_t(e)])] + 1);
        level[size_t(k)] = lv;
        depth = std::max(depth, lv + 1);
    }
    LevelSchedule s;
    s.level_ptr.assign(size_t(depth) + 1, 0);
    for (int64_t k = 0; k < n; ++k) ++s.level_ptr[size_t(level[size_t(k)]) + 1];
    for (int32_t d = 0; d < depth; ++d) s.level_ptr[size_t(d) + 1] += s.level_ptr[size_t(d)];
    s.rows.assign(size_t(n), 0);
    std::vector<int32_t> cur(s.level_ptr.begin(), s.level_ptr.end() - 1);
    for (int64_t k = n - 1; k >= 0; --k) s.rows[size_t(cur[size_t(level[size_t(k)])]++)] = int32_t(k);
    return s;
}

namespace {

// column j of a triangular inverse into `out` (index, value), increasing index
template <bool Upper>
void inverse_column(const std::vector<std::vector<std::pair<int32_t, double>>>& cols, const std::vector<double>& pivot,
                    int32_t j, std::vector<double>& acc, std::vector<char>& mark,
                    std::vector<std::pair<int32_t, double>>& out) {
    // min-heap (L: increasing index) or max-heap (U: decreasing) of touched rows
    std::vector<int32_t> heap;
    auto before = [](int32_t a, int32_t b) { return Upper ? a < b : a > b; };
    auto touch = [&](int32_t i) {
        if (!mark[size_t(i)]) {
            mark[size_t(i)] = 1;
            acc[size_t(i)] = 0.0;
            heap.push_back(i);
            std::push_heap(heap.begin(), heap.end(), before);
        }
    };
    touch(j);
    acc[size_t(j)] = 1.0;
    double biggest = 0.0;
    out.clear();
    const double rel = std::ldexp(1.0, -60);
    while (!heap.empty()) {
        std::pop_heap(heap.begin(), heap.end(), before);
        const int32_t i = heap.back();
        heap.pop_back();
        mark[size_t(i)] = 0;
        double x = acc[size_t(i)];
        if (Upper) x = x / pivot[size_t(i)];
        biggest = std::max(biggest, std::fabs(x));
        if (!(std::fabs(x) >= rel * biggest)) continue;  // dropped, not propagated
        out.emplace_back(i, x);
        // propagate to the rows that column i of the factor reaches
        for (const auto& e : cols[size_t(i)]) {
            touch(e.first);
            acc[size_t(e.first)] -= e.second * x;
        }
    }
    std::sort(out.begin(), out.end());
}

}  // namespace

bool triangular_inverses(const CsrRows& lower, const CsrRows& upper, const std::vector<double>& pivot, int64_t cap,
                         CsrRows& linv, CsrRows& uinv) {
    const int64_t n = lower.n;
    const size_t nn = static_cast<size_t>(n);
    // the factors by columns
    std::vector<std::vector<std::pair<int32_t, double>>> lcols(nn), ucols(nn);
    for (int64_t r = 0; r < n; ++r) {
        for (int64_t k = lower.ptr[size_t(r)]; k < lower.ptr[size_t(r) + 1]; ++k)
            lcols[size_t(lower.col[size_t(k)])].emplace_back(int32_t(r), lower.val[size_t(k)]);
        for (int64_t k = upper.ptr[size_t(r)]; k < upper.ptr[size_t(r) + 1]; ++k)
            ucols[size_t(upper.col[size_t(k)])].emplace_back(int32_t(r), upper.val[size_t(k)]);
    }
    // columns of the inverses, gathered into rows afterwards
    std::vector<std::vector<std::pair<int32_t, double>>> lrows(nn), urows(nn);
    std::vector<double> acc(nn, 0.0);
    std::vector<char> mark(nn, 0);
    std::vector<std::pair<int32_t, double>> col;
    int64_t total = 0;
    for (int64_t j = 0; j < n; ++j) {
        inverse_column<false>(lcols, pivot, int32_t(j), acc, mark, col);
        total += int64_t(col.size());
        for (const auto& e : col) lrows[size_t(e.first)].emplace_back(int32_t(j), e.second);
        inverse_column<true>(ucols, pivot, int32_t(j), acc, mark, col);
        total += int64_t(col.size());
        for (const auto& e : col) urows[size_t(e.first)].emplace_back(int32_t(j), e.second);
        if (total > cap) {
            linv = CsrRows();
            uinv = CsrRows();
            return false;
        }
    }
    for (auto* out : {&linv, &uinv}) {
        *out = CsrRows();
        out->n = n;
        out->ptr.assign(1, 0);
    }
    for (int64_t r = 0; r < n; ++r) {
        push_row(linv, lrows[size_t(r)]);  // columns increasing: j runs upwards
        push_row(uinv, urows[size_t(r)]);
    }
    return true;
}

CmdgfmFactor cmdgfm_factor(const CsrRows& m, int64_t np, double tau) {
    CmdgfmFactor f;
    f.np = np;
    f.nx = m.n - np;
    f.coupling.n = f.nx;
    f.coupling.ptr.assign(1, 0);
    for (int64_t r = np; r < m.n; ++r) {
        for (int64_t k = m.ptr[size_t(r)]; k < m.ptr[size_t(r) + 1]; ++k)
            if (m.col[size_t(k)] < np) {
                f.coupling.col.push_back(m.col[size_t(k)]);
                f.coupling.val.push_back(m.val[size_t(k)]);
            }
        f.coupling.ptr.push_back(int64_t(f.coupling.col.size()));
    }
    if (f.nx == 0) return f;
    f.schur = cmdgfm_schur(m, np);
    crout_ilu(f.schur, tau, f.lower, f.upper, f.pivot);
    f.lsched = forward_levels(f.lower);
    f.usched = backward_levels(f.upper);
    // the inverses, when they stay below 64 entries a row on average
    triangular_inverses(f.lower, f.upper, f.pivot, 64 * f.nx + 1024, f.linv, f.uinv);
    return f;
}

}  // namespace tpa
