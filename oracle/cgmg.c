/*
 * Oracle (test infrastructure only): C/OpenMP restatement of the solve loop of
 * TwoPhaseAMR.jl's pressure solve, used as the timed CPU baseline.  It consumes
 * the hierarchy built by the Python oracle (assembled level matrices, the
 * assembled smoothed prolongation P and its transpose, the augmented coarse
 * inverse) and runs exactly the reference's cycle:
 *
 *   src/solvers/multigrid/cycles.jl:8-24     `_smooth!` (damped Jacobi, means removed per sweep)
 *   src/solvers/multigrid/cycles.jl:46-77    `_vcycle!`
 *   src/solvers/multigrid/hierarchy.jl:208-246, 316-343  transfers, component projections
 *   src/operators/elliptic.jl:1125-1180      factorized action (CG operator)
 *   src/solvers/multigrid/elliptic_solver.jl:403-612  Krylov.jl cg! loop with the strong
 *                                             residual callback, restarts, targets
 *
 * Only tests/ and the CPU-baseline leg of bench.py load this code.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int64_t n;
    const int64_t* rp;
    const int32_t* ci;
    const double* v;       /* level matrix (row form) */
    const double* dinv;
    double w;
    const double* vol;
    const int32_t* slot;   /* component slot or -1 */
    int32_t ncomp;
    const double* cvol;
    /* transfer to the next level */
    const int64_t* prp;    /* P rows (fine) */
    const int32_t* pci;
    const double* pv;
    const int64_t* trp;    /* P' rows (coarse) */
    const int32_t* tci;
    const double* tv;
    double *x, *b, *t, *r; /* work */
} cg_level;

typedef struct {
    int64_t nc, nf;
    const int32_t* fm;
    const int32_t* fp;
    const double* area;
    const double* sk;
    const int64_t* kp;     /* K CSR over faces */
    const int32_t* ki;
    const double* kv;
    const int64_t* inc_off;  /* cell -> faces */
    const int32_t* inc_face;
    const int8_t* inc_sign;
    double *fin, *fout;
} cg_fine;

typedef struct {
    int32_t cycles, converged;
    double initial_linf, final_linf, target;
} cg_stats;

static void spmv(int64_t n, const int64_t* rp, const int32_t* ci, const double* v, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        double a = 0;
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) a += v[k] * x[ci[k]];
        y[i] = a;
    }
}

static void fine_apply(const cg_fine* F, const double* x, double* y) {
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < F->nf; ++f) F->fin[f] = F->sk[f] * F->area[f] * (x[F->fp[f]] - x[F->fm[f]]);
    spmv(F->nf, F->kp, F->ki, F->kv, F->fin, F->fout);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < F->nc; ++c) {
        double a = 0;
        for (int64_t k = F->inc_off[c]; k < F->inc_off[c + 1]; ++k) {
            int32_t f = F->inc_face[k];
            a += F->inc_sign[k] * F->area[f] * F->sk[f] * F->fout[f];
        }
        y[c] = a;
    }
}

static double dot(int64_t n, const double* a, const double* b) {
    double s = 0;
#pragma omp parallel for schedule(static) reduction(+ : s)
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

static double strong_max(int64_t n, const double* r, const double* vol) {
    double m = 0;
#pragma omp parallel for schedule(static) reduction(max : m)
    for (int64_t i = 0; i < n; ++i)
        if (vol[i] > 0) {
            double q = fabs(r[i]) / vol[i];
            if (q > m || q != q) m = q;
        }
    return m;
}

static void comp_sums(const cg_level* L, const double* v, int weighted, double* sums) {
    for (int s = 0; s < L->ncomp; ++s) {
        double a = 0;
#pragma omp parallel for schedule(static) reduction(+ : a)
        for (int64_t i = 0; i < L->n; ++i)
            if (L->slot[i] == s) a += weighted ? L->vol[i] * v[i] : v[i];
        sums[s] = a / L->cvol[s];
    }
}

static void remove_means(const cg_level* L, double* x) {
    double sums[64];
    comp_sums(L, x, 1, sums);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < L->n; ++i)
        if (L->slot[i] >= 0) x[i] -= sums[L->slot[i]];
}

static void project_rhs(const cg_level* L, double* b) {
    double sums[64];
    comp_sums(L, b, 0, sums);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < L->n; ++i)
        if (L->slot[i] >= 0) b[i] -= L->vol[i] * sums[L->slot[i]];
}

static void smooth(cg_level* L, int sweeps) {
    for (int s = 0; s < sweeps; ++s) {
        spmv(L->n, L->rp, L->ci, L->v, L->x, L->t);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < L->n; ++i) L->x[i] += L->w * L->dinv[i] * (L->b[i] - L->t[i]);
        if (L->ncomp) remove_means(L, L->x);
    }
}

typedef struct {
    int nlevels, pre, post;
    cg_level* lv;
    const double* cinv;
    int64_t cn;
} cg_mg;

static void vcycle(cg_mg* M, int l) {
    cg_level* L = &M->lv[l];
    if (L->ncomp) project_rhs(L, L->b);
    if (l == M->nlevels - 1) {
        const int64_t n = M->cn;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            double a = 0;
            for (int64_t k = 0; k < n; ++k) a += M->cinv[i * n + k] * L->b[k];
            L->x[i] = a;
        }
        return;
    }
    memset(L->x, 0, sizeof(double) * (size_t)L->n);
    smooth(L, M->pre);
    spmv(L->n, L->rp, L->ci, L->v, L->x, L->t);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < L->n; ++i) L->r[i] = L->b[i] - L->t[i];
    cg_level* C = &M->lv[l + 1];
    spmv(C->n, L->trp, L->tci, L->tv, L->r, C->b);
    vcycle(M, l + 1);
    spmv(L->n, L->prp, L->pci, L->pv, C->x, L->t);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < L->n; ++i) L->x[i] += L->t[i];
    if (L->ncomp) remove_means(L, L->x);
    smooth(L, M->post);
}

static void precondition(cg_mg* M, const double* r, double* z) {
    cg_level* L = &M->lv[0];
    memcpy(L->b, r, sizeof(double) * (size_t)L->n);
    vcycle(M, 0);
    memcpy(z, L->x, sizeof(double) * (size_t)L->n);
}

/* abs bound of the factorized action, for the roundoff floor (cycles.jl:108-179) */
static double roundoff_floor(const cg_fine* F, const double* x, const double* b, const double* vol, double* tmp) {
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < F->nf; ++f) F->fin[f] = F->sk[f] * F->area[f] * (fabs(x[F->fm[f]]) + fabs(x[F->fp[f]]));
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < F->nf; ++f) {
        double a = 0;
        for (int64_t k = F->kp[f]; k < F->kp[f + 1]; ++k) a += fabs(F->kv[k]) * F->fin[F->ki[k]];
        F->fout[f] = F->area[f] * F->sk[f] * a;
    }
    double scale = 0;
#pragma omp parallel for schedule(static) reduction(max : scale)
    for (int64_t c = 0; c < F->nc; ++c) {
        double a = 0;
        for (int64_t k = F->inc_off[c]; k < F->inc_off[c + 1]; ++k) a += F->fout[F->inc_face[k]];
        tmp[c] = a;
        if (vol[c] > 0) {
            double q = fmax(a / vol[c], fabs(b[c]) / vol[c]);
            if (q > scale) scale = q;
        }
    }
    return 128 * 2.220446049250313e-16 * fmax(1.0, scale);
}

static double guarded(const cg_fine* F, const double* x, const double* b, const double* vol, double* tmp,
                      double target, double init, double cur) {
    if (!(isfinite(init) && isfinite(cur) && target < cur && cur < init)) return target;
    double fl = roundoff_floor(F, x, b, vol, tmp);
    return (isfinite(fl) && fl < init / 100) ? fmax(target, fl) : target;
}

int cgmg_solve(int nlevels, cg_level* levels, cg_fine* F, const double* cinv, int64_t cn, int pre, int post,
               const double* rhs_strong, double* x, double rtol, double atol, int max_cycles, int threads,
               cg_stats* st) {
    if (threads > 0) omp_set_num_threads(threads);
    const double eps = 2.220446049250313e-16;
    cg_mg M = {nlevels, pre, post, levels, cinv, cn};
    cg_level* L0 = &levels[0];
    const int64_t n = L0->n;
    const double* vol = L0->vol;
    double* b = malloc(sizeof(double) * (size_t)n);
    double* r = malloc(sizeof(double) * (size_t)n);
    double* z = malloc(sizeof(double) * (size_t)n);
    double* p = malloc(sizeof(double) * (size_t)n);
    double* ap = malloc(sizeof(double) * (size_t)n);
    double* xc = malloc(sizeof(double) * (size_t)n);
    double* tmp = malloc(sizeof(double) * (size_t)n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        if (vol[i] == 0) {
            b[i] = 0;
            x[i] = 0;
        } else
            b[i] = rhs_strong[i] * vol[i];
    }
    if (L0->ncomp) {
        project_rhs(L0, b);
        remove_means(L0, x);
    }
    fine_apply(F, x, tmp);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - tmp[i];
    double init = strong_max(n, r, vol);
    double floor = roundoff_floor(F, x, b, vol, tmp);
    double target = fmax(atol, fmax(rtol * fmax(init, eps), floor));
    int total = 0;
    if (init > target) {
        while (total < max_cycles) {
            /* Krylov.jl cg!, warm start at x */
            memset(xc, 0, sizeof(double) * (size_t)n);
            fine_apply(F, x, tmp);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) r[i] = b[i] - tmp[i];
            precondition(&M, r, z);
            memcpy(p, z, sizeof(double) * (size_t)n);
            double gamma = dot(n, r, z), pnorm2 = gamma;
            int it = 0, itmax = max_cycles - total, stop = gamma == 0 || itmax <= 0;
            while (!stop) {
                fine_apply(F, p, ap);
                double pAp = dot(n, p, ap);
                if (pAp <= eps * pnorm2 && fabs(pAp) <= eps * pnorm2) break;
                double alpha = gamma / pAp;
#pragma omp parallel for schedule(static)
                for (int64_t i = 0; i < n; ++i) {
                    xc[i] += alpha * p[i];
                    r[i] -= alpha * ap[i];
                }
                precondition(&M, r, z);
                double gn = dot(n, r, z);
                double rnorm = sqrt(gn);
                int solved = rnorm + 1.0 <= 1.0;
                if (!solved) {
                    double beta = gn / gamma;
                    pnorm2 = gn + beta * beta * pnorm2;
                    gamma = gn;
#pragma omp parallel for schedule(static)
                    for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
                }
                ++it;
                stop = solved || it >= itmax || strong_max(n, r, vol) <= target;
            }
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) x[i] += xc[i];
            total += it;
            if (L0->ncomp) remove_means(L0, x);
            fine_apply(F, x, tmp);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) r[i] = b[i] - tmp[i];
            double fin = strong_max(n, r, vol);
            double eff = guarded(F, x, b, vol, tmp, target, init, fin);
            if (fin <= eff) break;
            if (!isfinite(fin) || it == 0) break;
        }
    }
    if (L0->ncomp) remove_means(L0, x);
    fine_apply(F, x, tmp);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - tmp[i];
    double fin = strong_max(n, r, vol);
    target = guarded(F, x, b, vol, tmp, target, init, fin);
    st->cycles = total;
    st->converged = isfinite(fin) && isfinite(target) && fin <= target;
    st->initial_linf = init;
    st->final_linf = fin;
    st->target = target;
    free(b); free(r); free(z); free(p); free(ap); free(xc); free(tmp);
    return 0;
}
