/*
 * fgmres_oracle.c -- CPU restatement, in FP64 with OpenMP over rows, of the
 * library's convergent Poisson solve (TEST INFRASTRUCTURE ONLY: the checker
 * that tests/ compare the GPU solve with, and the CPU baseline that bench.py
 * times; nothing on the product path links or calls it).
 *
 * The reference's own multigrid_Poisson_solver (fractional_step_solver.h:
 * 150-246) runs a fixed number of V-cycles and never reaches a tolerance; the
 * system it aims at -- lap_Poison with row 0 replaced by the pin p[0] = 0,
 * which its relaxation re-imposes after every sweep (:180-183) -- is solved
 * here to a relative residual, with the design of the library's solver:
 *   - per level the pinned operator; a Chebyshev polynomial in D^-1 A on
 *     interior rows (interval [lmax / ratio, 1.05 lmax], lmax by 40 steps of
 *     power iteration from a fixed hashed start vector), the boundary rows
 *     solved exactly after every step (a boundary row couples only to itself
 *     and interior nodes);
 *   - restriction of the interior residual with create_restriction_matrix's
 *     interpolation weights (mesh_functions.h:533-600) on every non-boundary
 *     coarse row except the pinned one; prolongation with
 *     create_prolongation_matrix's weights (:602-670) on every fine row,
 *     shifted so that the pinned node takes no correction;
 *   - the coarsest level by its dense inverse (Gauss-Jordan with partial
 *     pivoting);
 *   - flexible GMRES(m) in FP64 right-preconditioned by one V-cycle: classical
 *     Gram-Schmidt with a second pass when the first cancelled more than
 *     1 - 1/sqrt(2) of |w| (Daniel-Gragg-Kaufman-Stewart), Givens rotations,
 *     at most five restart cycles.
 * Row sums run in slot order; dot products are OpenMP reductions (their
 * summation order depends on the thread count, so results agree with the GPU
 * to the solve's tolerance, not bit for bit).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define CS_EXPORT __attribute__((visibility("default")))
#define CS_MAX_KRYLOV 128

typedef struct {
    int n, k;
    const int *cloud;            /* [n][k], slot 0 the row itself */
    double *A;                   /* pinned operator [n][k] */
    double *dinv;
    const unsigned char *btag;
    int *bnd;                    /* boundary rows */
    int nbnd;
    int kr;                      /* restriction into this level: [n][kr] over cloud_{l-1}[rpts[i]] */
    const int *rpts;
    const double *rw;
    int kp;                      /* prolongation into this level: [n][kp] over cloud_{l+1}[ppts[i]] */
    const int *ppts;
    const double *pw;
    double lmax;
    double *r, *e, *e2, *d, *q;
} cs_level;

typedef struct {
    int nl;
    cs_level *L;
    double *cinv;                /* dense inverse of the coarsest pinned operator */
} cs_ctx;

CS_EXPORT void *orc_cs_new(int nl)
{
    cs_ctx *c = (cs_ctx *)calloc(1, sizeof(cs_ctx));
    c->nl = nl;
    c->L = (cs_level *)calloc((size_t)nl, sizeof(cs_level));
    return c;
}

CS_EXPORT void orc_cs_free(void *h)
{
    cs_ctx *c = (cs_ctx *)h;
    for (int l = 0; l < c->nl; l++) {
        cs_level *L = &c->L[l];
        free(L->A); free(L->dinv); free(L->bnd);
        free(L->r); free(L->e); free(L->e2); free(L->d); free(L->q);
    }
    free(c->cinv);
    free(c->L);
    free(c);
}

/* One level: cloud and lap_Poison [n][k] (row-major), boundary tags, and the
 * solver's transfer weights into this level (restr [n][kr] over the finer
 * level's cloud at rpts, NULL on level 0; prol [n][kp] over the coarser
 * level's cloud at ppts, NULL on the coarsest).  The arrays must outlive the
 * context; lapP is copied (row 0 pinned). */
CS_EXPORT void orc_cs_level(void *h, int l, int n, int k, const int *cloud, const double *lapP,
                            const unsigned char *btag, int kr, const int *rpts, const double *restr, int kp,
                            const int *ppts, const double *prol)
{
    cs_ctx *c = (cs_ctx *)h;
    cs_level *L = &c->L[l];
    L->n = n; L->k = k; L->cloud = cloud; L->btag = btag;
    L->kr = kr; L->rpts = rpts; L->rw = restr;
    L->kp = kp; L->ppts = ppts; L->pw = prol;
    L->A = (double *)malloc(sizeof(double) * (size_t)n * k);
    memcpy(L->A, lapP, sizeof(double) * (size_t)n * k);
    for (int j = 0; j < k; j++) L->A[j] = j == 0 ? 1.0 : 0.0;   /* the pin p[0] = 0 */
    L->dinv = (double *)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) L->dinv[i] = 1.0 / L->A[(size_t)i * k];
    L->nbnd = 0;
    L->bnd = (int *)malloc(sizeof(int) * (size_t)n);
    for (int i = 0; i < n; i++) if (btag[i]) L->bnd[L->nbnd++] = i;
    double **v[5] = {&L->r, &L->e, &L->e2, &L->d, &L->q};
    for (int t = 0; t < 5; t++) *v[t] = (double *)calloc((size_t)n, sizeof(double));
}

static inline double row_dot(const cs_level *L, const double *x, int i)
{
    const double *a = L->A + (size_t)i * L->k;
    const int *cl = L->cloud + (size_t)i * L->k;
    double s = 0.0;
    for (int j = 0; j < L->k; j++) s += a[j] * x[cl[j]];
    return s;
}

static double dot(int n, const double *a, const double *b)
{
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

/* spectral radius of D^-1 A on interior rows: 40 power steps */
static double estimate_lmax(cs_level *L)
{
    const int n = L->n;
    double *v = (double *)malloc(sizeof(double) * (size_t)n), *w = (double *)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) {
        unsigned hh = (unsigned)i * 2654435761u;
        hh ^= hh >> 16; hh *= 2246822519u; hh ^= hh >> 13;
        v[i] = L->btag[i] ? 0.0 : ((double)(hh & 0xffffff) / 16777216.0 - 0.5);
    }
    double lam = 0.0;
    for (int it = 0; it < 40; it++) {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) w[i] = L->btag[i] ? 0.0 : L->dinv[i] * row_dot(L, v, i);
        const double sq = dot(n, w, w);
        if (it > 0) lam = sqrt(sq);
        const double sc = sq > 0 ? 1.0 / sqrt(sq) : 0.0;
        for (int i = 0; i < n; i++) v[i] = w[i] * sc;
    }
    free(v); free(w);
    return lam > 0 && isfinite(lam) ? lam : 2.0;
}

/* dense inverse of the coarsest pinned operator: Gauss-Jordan, partial pivoting */
static double *dense_inverse(const cs_level *L)
{
    const int n = L->n;
    double *M = (double *)calloc((size_t)n * 2 * n, sizeof(double));
    for (int i = 0; i < n; i++) {
        for (int j = 0; j < L->k; j++) M[(size_t)i * 2 * n + L->cloud[(size_t)i * L->k + j]] += L->A[(size_t)i * L->k + j];
        M[(size_t)i * 2 * n + n + i] = 1.0;
    }
    for (int col = 0; col < n; col++) {
        int pr = col;
        for (int r = col + 1; r < n; r++)
            if (fabs(M[(size_t)r * 2 * n + col]) > fabs(M[(size_t)pr * 2 * n + col])) pr = r;
        if (pr != col)
            for (int c = 0; c < 2 * n; c++) {
                double t = M[(size_t)col * 2 * n + c];
                M[(size_t)col * 2 * n + c] = M[(size_t)pr * 2 * n + c];
                M[(size_t)pr * 2 * n + c] = t;
            }
        const double piv = M[(size_t)col * 2 * n + col];
        for (int c = 0; c < 2 * n; c++) M[(size_t)col * 2 * n + c] /= piv;
#pragma omp parallel for schedule(static)
        for (int r = 0; r < n; r++) {
            if (r == col) continue;
            const double f = M[(size_t)r * 2 * n + col];
            if (f != 0.0)
                for (int c = 0; c < 2 * n; c++) M[(size_t)r * 2 * n + c] -= f * M[(size_t)col * 2 * n + c];
        }
    }
    double *inv = (double *)malloc(sizeof(double) * (size_t)n * n);
    for (int i = 0; i < n; i++) memcpy(inv + (size_t)i * n, M + (size_t)i * 2 * n + n, sizeof(double) * (size_t)n);
    free(M);
    return inv;
}

CS_EXPORT void orc_cs_prepare(void *h)
{
    cs_ctx *c = (cs_ctx *)h;
    for (int l = 0; l < c->nl - 1; l++) c->L[l].lmax = estimate_lmax(&c->L[l]);
    free(c->cinv);
    c->cinv = dense_inverse(&c->L[c->nl - 1]);
}

/* boundary rows solved exactly given the interior values of e */
static void boundary_exact(cs_level *L, double *e)
{
#pragma omp parallel for schedule(static)
    for (int t = 0; t < L->nbnd; t++) {
        const int i = L->bnd[t];
        e[i] = e[i] + (L->r[i] - row_dot(L, e, i)) * L->dinv[i];
    }
}

static void smooth(cs_level *L, int deg, double ratio, int zero_start)
{
    const int n = L->n;
    const double lM = 1.05 * L->lmax, lm = L->lmax / ratio;
    const double th = 0.5 * (lM + lm), de = 0.5 * (lM - lm), sig = th / de;
    double rho = 1.0 / sig;
    if (zero_start) {
        for (int i = 0; i < n; i++) L->e[i] = L->btag[i] ? L->r[i] * L->dinv[i] : 0.0;
    } else {
        boundary_exact(L, L->e);
    }
    for (int step = 0; step < deg; step++) {
        double c1 = 0.0, c2;
        if (step == 0) c2 = 1.0 / th;
        else {
            const double rn = 1.0 / (2.0 * sig - rho);
            c1 = rn * rho;
            c2 = 2.0 * rn / de;
            rho = rn;
        }
        double *e = L->e, *eo = L->e2;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
            if (L->btag[i]) { eo[i] = e[i]; continue; }
            const double q = L->r[i] - row_dot(L, e, i);
            const double di = step == 0 ? c2 * L->dinv[i] * q : c1 * L->d[i] + c2 * L->dinv[i] * q;
            L->d[i] = di;
            eo[i] = e[i] + di;
        }
        L->e = eo; L->e2 = e;
        boundary_exact(L, L->e);
    }
}

static void vcycle(cs_ctx *c, int l, int deg, double ratio)
{
    cs_level *L = &c->L[l];
    if (l == c->nl - 1) {
        const int n = L->n;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
            double s = 0.0;
            for (int j = 0; j < n; j++) s += c->cinv[(size_t)i * n + j] * L->r[j];
            L->e[i] = s;
        }
        return;
    }
    smooth(L, deg, ratio, 1);
    const int n = L->n;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) L->q[i] = L->btag[i] ? 0.0 : L->r[i] - row_dot(L, L->e, i);
    cs_level *C = &c->L[l + 1];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < C->n; i++) {
        if (C->btag[i] || i == 0) { C->r[i] = 0.0; continue; }
        const int *cl = L->cloud + (size_t)C->rpts[i] * L->k;
        const double *w = C->rw + (size_t)i * C->kr;
        double s = 0.0;
        for (int j = 0; j < C->kr; j++) s += w[j] * L->q[cl[j]];
        C->r[i] = s;
    }
    vcycle(c, l + 1, deg, ratio);
    double shift = 0.0;
    {
        const int *cl = C->cloud + (size_t)L->ppts[0] * C->k;
        for (int j = 0; j < L->kp; j++) shift += L->pw[j] * C->e[cl[j]];
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
        const int *cl = C->cloud + (size_t)L->ppts[i] * C->k;
        const double *w = L->pw + (size_t)i * L->kp;
        double s = 0.0;
        for (int j = 0; j < L->kp; j++) s += w[j] * C->e[cl[j]];
        L->e[i] += s - shift;
    }
    smooth(L, deg, ratio, 0);
}

/* FGMRES(m) on the pinned level-0 system A p = b (b[0] taken as 0), p the
 * initial guess.  Returns 0 on convergence to rel_tol (|b - A p| / |b| over
 * the pinned system), 1 otherwise; *iters = V-cycles, *relres the last true
 * relative residual. */
CS_EXPORT int orc_cs_solve(void *h, const double *b_in, double *p, double tol, int max_iters, int deg, double ratio,
                           int *iters, double *relres)
{
    cs_ctx *c = (cs_ctx *)h;
    cs_level *L0 = &c->L[0];
    const int n = L0->n;
    int m = max_iters < CS_MAX_KRYLOV ? max_iters : CS_MAX_KRYLOV;
    double *b = (double *)malloc(sizeof(double) * (size_t)n);
    memcpy(b, b_in, sizeof(double) * (size_t)n);
    b[0] = 0.0;
    double *V = (double *)malloc(sizeof(double) * (size_t)(m + 1) * n);
    double *Z = (double *)malloc(sizeof(double) * (size_t)m * n);
    double *H = (double *)calloc((size_t)(m + 1) * m, sizeof(double));
    double cs[CS_MAX_KRYLOV], sn[CS_MAX_KRYLOV], g[CS_MAX_KRYLOV + 1], y[CS_MAX_KRYLOV];
    double h1[CS_MAX_KRYLOV + 2], h2[CS_MAX_KRYLOV + 2];
    const double bnorm = sqrt(dot(n, b, b));
    int total = 0, ok = 0;
    double rr = 1.0;
    for (int restart = 0; restart <= 4; restart++) {
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) V[i] = b[i] - row_dot(L0, p, i);
        const double beta = sqrt(dot(n, V, V));
        rr = bnorm > 0 ? beta / bnorm : 0.0;
        if (!isfinite(rr)) break;
        if (bnorm == 0 || rr < tol) { ok = 1; break; }
        for (int i = 0; i < n; i++) V[i] /= beta;
        memset(g, 0, sizeof(g));
        g[0] = beta;
        int jd = 0;
        for (int j = 0; j < m; j++) {
            memcpy(L0->r, V + (size_t)j * n, sizeof(double) * (size_t)n);
            vcycle(c, 0, deg, ratio);
            memcpy(Z + (size_t)j * n, L0->e, sizeof(double) * (size_t)n);
            double *w = V + (size_t)(j + 1) * n;
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; i++) w[i] = row_dot(L0, Z + (size_t)j * n, i);
            for (int t = 0; t <= j + 1; t++) h1[t] = dot(n, V + (size_t)t * n, w);
            for (int t = 0; t <= j; t++) h2[t] = 0.0;
            for (int t = 0; t <= j; t++) {
                const double *vt = V + (size_t)t * n;
#pragma omp parallel for schedule(static)
                for (int i = 0; i < n; i++) w[i] -= h1[t] * vt[i];
            }
            double nrm = dot(n, w, w);
            if (nrm < 0.5 * h1[j + 1]) {
                for (int t = 0; t <= j; t++) h2[t] = dot(n, V + (size_t)t * n, w);
                for (int t = 0; t <= j; t++) {
                    const double *vt = V + (size_t)t * n;
#pragma omp parallel for schedule(static)
                    for (int i = 0; i < n; i++) w[i] -= h2[t] * vt[i];
                }
                nrm = dot(n, w, w);
            }
            const double wn = sqrt(nrm > 0 ? nrm : 0.0);
            for (int i = 0; i < n; i++) w[i] = wn > 0 ? w[i] / wn : 0.0;
            double *col = H + (size_t)j * (m + 1);
            for (int t = 0; t <= j; t++) col[t] = h1[t] + h2[t];
            col[j + 1] = wn;
            for (int t = 0; t < j; t++) {
                const double t0 = cs[t] * col[t] + sn[t] * col[t + 1];
                col[t + 1] = -sn[t] * col[t] + cs[t] * col[t + 1];
                col[t] = t0;
            }
            const double rden = hypot(col[j], col[j + 1]);
            cs[j] = rden > 0 ? col[j] / rden : 1.0;
            sn[j] = rden > 0 ? col[j + 1] / rden : 0.0;
            col[j] = rden;
            col[j + 1] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            total++;
            jd = j + 1;
            const double est = fabs(g[j + 1]) / bnorm;
            if (!isfinite(est) || est < tol) break;
        }
        for (int t = jd - 1; t >= 0; t--) {
            double s = g[t];
            for (int q = t + 1; q < jd; q++) s -= H[(size_t)q * (m + 1) + t] * y[q];
            y[t] = s / H[(size_t)t * (m + 1) + t];
        }
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
            double s = p[i];
            for (int t = 0; t < jd; t++) s += y[t] * Z[(size_t)t * n + i];
            p[i] = s;
        }
    }
    if (!ok) {
        /* the last cycle's update has not been checked yet */
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) V[i] = b[i] - row_dot(L0, p, i);
        rr = bnorm > 0 ? sqrt(dot(n, V, V)) / bnorm : 0.0;
        ok = rr < tol;
    }
    free(b); free(V); free(Z); free(H);
    *iters = total;
    *relres = rr;
    return ok ? 0 : 1;
}
