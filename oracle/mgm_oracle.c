/*
 * mgm_oracle.c -- CPU restatement of the reference solver's hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing on the product path links, loads or calls
 * this file; it is the checker that tests/, __graft_entry__.smoke() and the
 * bench's cpu_baseline leg compare the CUDA path against.  Parity of this
 * restatement is pinned against the reference's own code compiled from its
 * sources (oracle/ref_shim.c -> oracle/_ref/libref.so) by tests/test_oracle_pin.py
 * and against the committed fixtures in tests/golden/.
 *
 * Layout: every per-node stencil quantity is row-major [n][k] (the reference's
 * jagged `double**` rows laid end to end).  Built with -ffp-contract=off so the
 * rounding sequence of every sum and product is the one the reference's C code
 * performs under gcc on x86-64 (no FMA contraction).
 *
 * Exact-tie rule: the reference keeps, among equal distances, the one its kd
 * range search happens to list first (kdtree_functions.h:86-96, kdtree.c:812-830).
 * This restatement (and the CUDA path) orders candidates by (distance, index);
 * the two agree whenever no two candidates of a query share a distance bit for
 * bit, which the tests count.
 */
#include <math.h>
#include <stdio.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_EXPORT __attribute__((visibility("default")))

/* Built twice (oracle/Makefile): liboracle.so calls libm's pow() exactly as the
 * reference does (rbf.h:35-39, 68-72; mesh_functions.h:585-587) and is pinned
 * bit for bit against the reference; liboracle_crpow.so (-DORC_CR_POW) takes
 * the correctly rounded power instead, evaluated in binary128 and rounded once,
 * which is what the CUDA path computes (libm's pow is off by one ulp in about
 * 0.08% of calls, which no GPU code can reproduce). */
#ifdef ORC_CR_POW
#include <quadmath.h>
static double orc_pow(double x, double y)
{
    if (y == 0) return 1.0;
    __float128 q = x;
    if (y == (int)y) {
        __float128 r = q;
        for (int i = 1; i < (int)y; i++) r *= q;
        return (double)r;
    }
    int m = (int)(y - 0.5); /* y = m + 1/2 */
    __float128 r = sqrtq(q);
    for (int i = 0; i < m; i++) r *= q;
    return (double)r;
}
#define pow(x, y) orc_pow((x), (y))
#endif

/* ------------------------------------------------------------------------ */
/* kNN clouds: find_cloud_index / find_neighbours / find_nearest_point       */
/* kdtree_functions.h:28-35 (distance), 61-111 (top-k), 113-151, 153-175     */
/* ------------------------------------------------------------------------ */

typedef struct {
    int dim, ncx, ncy, ncz;
    double x0, y0, z0, cell;
    int *start;   /* ncells+1 */
    int *items;   /* node ids sorted by cell */
} grid_t;

static void grid_build(grid_t *g, int n, const double *x, const double *y, const double *z,
                       const unsigned char *mask, int dim)
{
    double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300, zmin = 1e300, zmax = -1e300;
    int cnt = 0;
    for (int i = 0; i < n; i++) {
        if (mask && !mask[i]) continue;
        cnt++;
        if (x[i] < xmin) xmin = x[i];
        if (x[i] > xmax) xmax = x[i];
        if (y[i] < ymin) ymin = y[i];
        if (y[i] > ymax) ymax = y[i];
        if (z[i] < zmin) zmin = z[i];
        if (z[i] > zmax) zmax = z[i];
    }
    if (cnt == 0) { xmin = xmax = ymin = ymax = zmin = zmax = 0; }
    double ex = xmax - xmin, ey = ymax - ymin, ez = zmax - zmin;
    double vol = dim == 3 ? fmax(ex, 1e-300) * fmax(ey, 1e-300) * fmax(ez, 1e-300) : fmax(ex, 1e-300) * fmax(ey, 1e-300);
    double cell = dim == 3 ? cbrt(2.0 * vol / (cnt > 0 ? cnt : 1)) : sqrt(2.0 * vol / (cnt > 0 ? cnt : 1));
    if (!(cell > 0)) cell = 1.0;
    g->dim = dim; g->cell = cell; g->x0 = xmin; g->y0 = ymin; g->z0 = zmin;
    g->ncx = (int)(ex / cell) + 1; g->ncy = (int)(ey / cell) + 1; g->ncz = dim == 3 ? (int)(ez / cell) + 1 : 1;
    long nc = (long)g->ncx * g->ncy * g->ncz;
    g->start = (int *)calloc((size_t)nc + 1, sizeof(int));
    g->items = (int *)malloc(sizeof(int) * (size_t)(cnt > 0 ? cnt : 1));
    int *cid = (int *)malloc(sizeof(int) * (size_t)n);
    for (int i = 0; i < n; i++) {
        if (mask && !mask[i]) { cid[i] = -1; continue; }
        int cx = (int)((x[i] - xmin) / cell), cy = (int)((y[i] - ymin) / cell), cz = dim == 3 ? (int)((z[i] - zmin) / cell) : 0;
        if (cx >= g->ncx) cx = g->ncx - 1;
        if (cy >= g->ncy) cy = g->ncy - 1;
        if (cz >= g->ncz) cz = g->ncz - 1;
        cid[i] = (cz * g->ncy + cy) * g->ncx + cx;
        g->start[cid[i] + 1]++;
    }
    for (long c = 0; c < nc; c++) g->start[c + 1] += g->start[c];
    int *fill = (int *)malloc(sizeof(int) * (size_t)nc);
    memcpy(fill, g->start, sizeof(int) * (size_t)nc);
    for (int i = 0; i < n; i++) if (cid[i] >= 0) g->items[fill[cid[i]]++] = i;
    free(fill); free(cid);
}

static void grid_free(grid_t *g) { free(g->start); free(g->items); }

/* dist_sq of kdtree_functions.h:28-35 (3 coordinates, left to right), then sqrt (:84). */
static inline double ref_distance(double px, double py, double pz, double qx, double qy, double qz)
{
    double s = 0, d;
    d = px - qx; s += d * d;
    d = py - qy; s += d * d;
    d = pz - qz; s += d * d;
    return sqrt(s);
}

/* k smallest (distance, index) among grid members, ascending. */
static void grid_topk(const grid_t *g, const double *x, const double *y, const double *z,
                      double px, double py, double pz, int k, double *bd, int *bi)
{
    int have = 0;
    int cx = (int)((px - g->x0) / g->cell), cy = (int)((py - g->y0) / g->cell), cz = g->dim == 3 ? (int)((pz - g->z0) / g->cell) : 0;
    if (cx < 0) cx = 0;
    if (cy < 0) cy = 0;
    if (cz < 0) cz = 0;
    if (cx >= g->ncx) cx = g->ncx - 1;
    if (cy >= g->ncy) cy = g->ncy - 1;
    if (cz >= g->ncz) cz = g->ncz - 1;
    int rmax = g->ncx + g->ncy + g->ncz;
    for (int r = 0; r <= rmax; r++) {
        int zlo = g->dim == 3 ? cz - r : 0, zhi = g->dim == 3 ? cz + r : 0;
        for (int zz = zlo; zz <= zhi; zz++) {
            if (zz < 0 || zz >= g->ncz) continue;
            for (int yy = cy - r; yy <= cy + r; yy++) {
                if (yy < 0 || yy >= g->ncy) continue;
                for (int xx = cx - r; xx <= cx + r; xx++) {
                    if (xx < 0 || xx >= g->ncx) continue;
                    int ring = abs(xx - cx);
                    if (abs(yy - cy) > ring) ring = abs(yy - cy);
                    if (abs(zz - cz) > ring) ring = abs(zz - cz);
                    if (ring != r) continue;
                    int c = (zz * g->ncy + yy) * g->ncx + xx;
                    for (int t = g->start[c]; t < g->start[c + 1]; t++) {
                        int q = g->items[t];
                        double d = ref_distance(px, py, pz, x[q], y[q], z[q]);
                        if (have == k && (d > bd[k - 1] || (d == bd[k - 1] && q > bi[k - 1]))) continue;
                        int pos = have < k ? have : k - 1;
                        while (pos > 0 && (bd[pos - 1] > d || (bd[pos - 1] == d && bi[pos - 1] > q))) {
                            bd[pos] = bd[pos - 1]; bi[pos] = bi[pos - 1]; pos--;
                        }
                        bd[pos] = d; bi[pos] = q;
                        if (have < k) have++;
                    }
                }
            }
        }
        /* every point outside rings 0..r lies at least r*cell away */
        if (have == k && bd[k - 1] < ((double)r - 1e-3) * g->cell) break;
    }
    for (int t = have; t < k; t++) { bd[t] = 100.0; bi[t] = 0; }
}

/* find_cloud_index (kdtree_functions.h:113-151): nodes i >= nb get the k
 * nearest non-corner nodes (self first); nodes i < nb get [i] followed by the
 * k-1 nearest nodes whose boundary tag is false. */
ORC_EXPORT void orc_knn_cloud(int n, int nb, const double *x, const double *y, const double *z,
                              const unsigned char *btag, int k, int dim, int *cloud)
{
    grid_t gall, gint;
    unsigned char *interior = (unsigned char *)malloc((size_t)n);
    for (int i = 0; i < n; i++) interior[i] = btag[i] ? 0 : 1;
    grid_build(&gall, n, x, y, z, NULL, dim);
    grid_build(&gint, n, x, y, z, interior, dim);
    /* rows are independent: OpenMP threads share the grids, each its own scratch */
#pragma omp parallel
    {
        double *bd = (double *)malloc(sizeof(double) * (size_t)k);
        int *bi = (int *)malloc(sizeof(int) * (size_t)k);
#pragma omp for schedule(dynamic, 1024)
        for (int i = 0; i < n; i++) {
            int *row = cloud + (size_t)i * k;
            if (i >= nb) {
                grid_topk(&gall, x, y, z, x[i], y[i], z[i], k, bd, bi);
                for (int j = 0; j < k; j++) row[j] = bi[j];
            } else {
                grid_topk(&gint, x, y, z, x[i], y[i], z[i], k, bd, bi);
                row[0] = i;
                for (int j = 1; j < k; j++) row[j] = bi[j - 1];
            }
        }
        free(bd); free(bi);
    }
    free(interior);
    grid_free(&gall); grid_free(&gint);
}

/* Number of queries whose k-list holds two bit-identical distances (where the
 * reference's kd-tree order, not the index, decides the slot order). */
ORC_EXPORT long orc_count_ties(int n, int nb, const double *x, const double *y, const double *z, int k, const int *cloud)
{
    long ties = 0;
    for (int i = 0; i < n; i++) {
        const int *row = cloud + (size_t)i * k;
        int j0 = i < nb ? 1 : 0;
        for (int j = j0 + 1; j < k; j++) {
            double a = ref_distance(x[i], y[i], z[i], x[row[j - 1]], y[row[j - 1]], z[row[j - 1]]);
            double b = ref_distance(x[i], y[i], z[i], x[row[j]], y[row[j]], z[row[j]]);
            if (a == b) { ties++; break; }
        }
    }
    return ties;
}

/* find_nearest_point (kdtree_functions.h:153-175): nearest node of level 2 for each node of level 1. */
ORC_EXPORT void orc_nearest(int n1, const double *x1, const double *y1, const double *z1,
                            int n2, const double *x2, const double *y2, const double *z2, int dim, int *out)
{
    grid_t g;
    grid_build(&g, n2, x2, y2, z2, NULL, dim);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int i = 0; i < n1; i++) {
        double bd[1]; int bi[1];
        grid_topk(&g, x2, y2, z2, x1[i], y1[i], z1[i], 1, bd, bi);
        out[i] = bi[0];
    }
    grid_free(&g);
}

/* ------------------------------------------------------------------------ */
/* Reordering: rcm_reordering_with_boundarynodes (mesh_functions.h:774-872)  */
/* FIFO breadth-first order from node 0 over cloud slots 1..k-1.            */
/* Returns the number of nodes reached (n when the stencil graph is connected). */
/* ------------------------------------------------------------------------ */
ORC_EXPORT int orc_bfs_order(int n, int k, const int *cloud, int *queue1)
{
    unsigned char *vis = (unsigned char *)calloc((size_t)n, 1);
    int count = 0, head = 0;
    queue1[count++] = 0; vis[0] = 1;
    while (head < count) {
        int cur = queue1[head++];
        for (int j = 1; j < k; j++) {
            int nbr = cloud[(size_t)cur * k + j];
            if (!vis[nbr]) { vis[nbr] = 1; queue1[count++] = nbr; }
        }
    }
    free(vis);
    return count;
}

/* Applies the permutation the way mesh_functions.h:821-855 does: new node i is
 * old node queue1[i]; cloud entries are renumbered through queue2 (inverse). */
ORC_EXPORT void orc_apply_order(int n, int k, const int *queue1,
                                double *x, double *y, double *z, double *nx, double *ny, double *nz,
                                unsigned char *btag, int *cloud)
{
    int *q2 = (int *)malloc(sizeof(int) * (size_t)n);
    for (int i = 0; i < n; i++) q2[queue1[i]] = i;
    double *t = (double *)malloc(sizeof(double) * (size_t)n);
    double *arrs[6] = {x, y, z, nx, ny, nz};
    for (int a = 0; a < 6; a++) {
        for (int i = 0; i < n; i++) t[i] = arrs[a][queue1[i]];
        memcpy(arrs[a], t, sizeof(double) * (size_t)n);
    }
    unsigned char *tb = (unsigned char *)malloc((size_t)n);
    for (int i = 0; i < n; i++) tb[i] = btag[queue1[i]];
    memcpy(btag, tb, (size_t)n);
    int *tc = (int *)malloc(sizeof(int) * (size_t)n * k);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < k; j++) tc[(size_t)i * k + j] = q2[cloud[(size_t)queue1[i] * k + j]];
    memcpy(cloud, tc, sizeof(int) * (size_t)n * k);
    free(q2); free(t); free(tb); free(tc);
}

/* correct_normal_directions (mesh_functions.h:478-527) */
ORC_EXPORT void orc_correct_normals(int n, int k, const double *x, const double *y, const double *z,
                                    const unsigned char *btag, const int *cloud,
                                    double *nx, double *ny, double *nz)
{
    for (int i = 0; i < n; i++) {
        if (!btag[i]) continue;
        double xa = 0, ya = 0, za = 0;
        short count = 0;
        for (int j = k - 1; j > 0; j--) {
            int c = cloud[(size_t)i * k + j];
            if (!btag[c]) { xa += x[c]; ya += y[c]; za += z[c]; count++; if (count == 1) break; }
        }
        xa = xa / count; ya = ya / count; za = za / count;
        double dx = xa - x[i], dy = ya - y[i], dz = za - z[i];
        double dot = dx * nx[i] + dy * ny[i] + dz * nz[i];
        if (dot > 0) { nx[i] = -nx[i]; ny[i] = -ny[i]; nz[i] = -nz[i]; }
        double mag = sqrt(nx[i] * nx[i] + ny[i] * ny[i] + nz[i] * nz[i]);
        nx[i] = nx[i] / mag; ny[i] = ny[i] / mag; nz[i] = nz[i] / mag;
    }
}

/* calculate_avg_dx (mesh_functions.h:895-910) */
ORC_EXPORT double orc_avg_dx(int n, int k, int dim, const double *x, const double *y, const double *z,
                             const unsigned char *btag, const int *cloud)
{
    double s = 0;
    for (int i = 0; i < n; i++) {
        if (btag[i]) continue;
        int c = cloud[(size_t)i * k + 1];
        double dx = x[i] - x[c], dy = y[i] - y[c], dz = dim == 3 ? z[i] - z[c] : 0;
        s += sqrt(dx * dx + dy * dy + dz * dz);
    }
    return s / n;
}

/* calculate_dt (general_functions.h:34-41) with rho = 1, mu = rho/Re, nu = mu/rho
 * (mesh_functions.h:97-99). */
ORC_EXPORT double orc_dt(double d_avg, double Re, double courant)
{
    double rho = 1, mu = rho / Re, nu = mu / rho;
    double termd = 2 * nu / (d_avg * d_avg);
    double termc = 1 / d_avg;
    double dt = 0.5 / (termd + termc);
    return dt * courant;
}

/* ------------------------------------------------------------------------ */
/* RBF-FD weights (rbf.h, mat_lib.h)                                         */
/* ------------------------------------------------------------------------ */

/* monomial exponents in calculate_parameters order (mesh_functions.h:131-170) */
ORC_EXPORT int orc_monomials(int dim, int deg, short *px, short *py, short *pz)
{
    int c = 0;
    if (dim == 2) {
        for (int i = 0; i <= deg; i++)
            for (int j = 0; j <= deg - i; j++) { px[c] = i; py[c] = j; pz[c] = 0; c++; }
    } else {
        for (int i = 0; i <= deg; i++)
            for (int j = 0; j <= deg - i; j++)
                for (int l = 0; l <= deg - i - j; l++) { px[c] = i; py[c] = j; pz[c] = l; c++; }
    }
    return c;
}

/* calculate_phs_rbf (rbf.h:32-40) */
static double phs_rbf(const double *p1, const double *p2, int phs, int dim)
{
    double sum = 0;
    for (int i = 0; i < dim; i++) sum += pow(p1[i] - p2[i], 2);
    if (sum == 0) return 0;
    return pow(sum, phs * 0.5);
}

/* create_A_matrix_from_cloud_indices (rbf.h:42-77), A row-major N x N (N = m + np),
 * bottom-right block zero (create_matrix zero-fills, mat_lib.h:118-133). */
static void build_A(int m, int np, int dim, int phs, const int *cl, const double *x, const double *y, const double *z,
                    const short *px, const short *py, const short *pz, double *A)
{
    int N = m + np;
    memset(A, 0, sizeof(double) * (size_t)N * N);
    double seed[3] = {x[cl[0]], y[cl[0]], z[cl[0]]};
    for (int i = 0; i < m; i++) {
        double p1[3] = {x[cl[i]], y[cl[i]], z[cl[i]]};
        A[(size_t)i * N + i] = 0;
        for (int j = i + 1; j < m; j++) {
            double p2[3] = {x[cl[j]], y[cl[j]], z[cl[j]]};
            double v = phs_rbf(p1, p2, phs, dim);
            A[(size_t)i * N + j] = v; A[(size_t)j * N + i] = v;
        }
    }
    for (int i = 0; i < m; i++)
        for (int j = 0; j < np; j++) {
            double v = 1;
            if (px[j] != 0) v *= pow(x[cl[i]] - seed[0], px[j]);
            if (py[j] != 0) v *= pow(y[cl[i]] - seed[1], py[j]);
            if (pz[j] != 0) v *= pow(z[cl[i]] - seed[2], pz[j]);
            A[(size_t)i * N + j + m] = v; A[(size_t)(j + m) * N + i] = v;
        }
}

/* matrixInverse_Gauss_Jordan (mat_lib.h:423-491): one bubble pass on column 0,
 * then elimination without pivoting, then row scaling.  aug: N x 2N scratch. */
static void gauss_jordan(int N, const double *A, double *Ainv, double *aug, double **rows)
{
    for (int i = 0; i < N; i++) {
        rows[i] = aug + (size_t)i * 2 * N;
        for (int j = 0; j < N; j++) rows[i][j] = A[(size_t)i * N + j];
        for (int j = N; j < 2 * N; j++) rows[i][j] = (j == i + N) ? 1 : 0;
    }
    for (int i = N - 1; i > 0; i--)
        if (rows[i - 1][0] < rows[i][0]) { double *t = rows[i]; rows[i] = rows[i - 1]; rows[i - 1] = t; }
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) {
            if (j == i) continue;
            double t = rows[j][i] / rows[i][i];
            for (int c = 0; c < 2 * N; c++) rows[j][c] -= rows[i][c] * t;
        }
    for (int i = 0; i < N; i++) {
        double t = rows[i][i];
        for (int c = 0; c < 2 * N; c++) rows[i][c] = rows[i][c] / t;
    }
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++) Ainv[(size_t)i * N + j] = rows[i][j + N];
}

/* Row 0 of the operator matrices of rbf.h:79-270 at the seed (the only row
 * multiply_matrices' result is read from, rbf.h:294-296).  op: 0 gradx,
 * 1 grady, 2 gradz, 3 laplacian. */
static void operator_row0(int op, int m, int np, int dim, int phs, const int *cl,
                          const double *x, const double *y, const double *z,
                          const short *px, const short *py, const short *pz, double *L)
{
    int N = m + np;
    for (int j = 0; j < N; j++) L[j] = 0;
    double p1[3] = {x[cl[0]], y[cl[0]], z[cl[0]]};
    double seed[3] = {p1[0], p1[1], p1[2]};
    for (int j = 0; j < m; j++) {
        double p2[3] = {x[cl[j]], y[cl[j]], z[cl[j]]};
        if (op <= 2) L[j] = phs * (p1[op] - p2[op]) * phs_rbf(p1, p2, phs - 2, dim);
        else L[j] = phs * phs * phs_rbf(p1, p2, phs - 2, dim);
    }
    if (op == 0) {
        L[m] = 0;
        for (int j = 1; j < np; j++) {
            if (px[j] == 0) L[j + m] = 0;
            else {
                double v = px[j] * pow(p1[0] - seed[0], px[j] - 1);
                v *= pow(p1[1] - seed[1], py[j]);
                v *= pow(p1[2] - seed[2], pz[j]);
                L[j + m] = v;
            }
        }
    } else if (op == 1) {
        L[0] = 0; /* rbf.h:141 zeroes column 0, not column m */
        for (int j = 1; j < np; j++) {
            if (py[j] == 0) L[j + m] = 0;
            else {
                double v = py[j] * pow(p1[1] - seed[1], py[j] - 1);
                v = v * pow(p1[0] - seed[0], px[j]);
                v = v * pow(p1[2] - seed[2], pz[j]);
                L[j + m] = v;
            }
        }
    } else if (op == 2) {
        L[0] = 0;
        for (int j = 1; j < np; j++) {
            if (pz[j] == 0) L[j + m] = 0;
            else {
                double v = pz[j] * pow(p1[2] - seed[2], pz[j] - 1);
                v = v * pow(p1[1] - seed[1], py[j]);
                v = v * pow(p1[0] - seed[0], px[j]);
                L[j + m] = v;
            }
        }
    } else {
        double d0 = p1[0] - seed[0], d1 = p1[1] - seed[1], d2 = p1[2] - seed[2];
        for (int j = 0; j < np; j++) {
            double tx = 0, ty = 0, tz = 0;
            if (dim == 3) {
                if (px[j] > 1) { tx = px[j] * (px[j] - 1) * pow(d0, px[j] - 2); tx *= pow(d1, py[j]); tx *= pow(d2, pz[j]); }
                else if (py[j] > 1) { ty = py[j] * (py[j] - 1) * pow(d1, py[j] - 2); ty *= pow(d0, px[j]); ty *= pow(d2, pz[j]); }
                else if (pz[j] > 1) { tz = pz[j] * (pz[j] - 1) * pow(d2, pz[j] - 2); tz *= pow(d0, px[j]); tz *= pow(d1, py[j]); }
                L[j + m] = tx + ty + tz;
            } else {
                if (px[j] > 1) { tx = px[j] * (px[j] - 1) * pow(d0, px[j] - 2); tx *= pow(d1, py[j]); }
                else if (py[j] > 1) { ty = py[j] * (py[j] - 1) * pow(d1, py[j] - 2); ty *= pow(d0, px[j]); }
                L[j + m] = tx + ty;
            }
        }
    }
}

/* create_derivative_matrices (rbf.h:401-421) incl. create_laplacian_for_Poisson
 * (rbf.h:382-399).  Outputs [n][k]; Dz written only in 3D. */
ORC_EXPORT void orc_derivative_weights(int n, int k, int dim, int phs, int poly_degree,
                                       const double *x, const double *y, const double *z,
                                       const double *nx, const double *ny, const double *nz,
                                       const unsigned char *btag, const int *cloud,
                                       double *Dx, double *Dy, double *Dz, double *lap, double *lapP)
{
    short px[64], py[64], pz[64];
    int np = orc_monomials(dim, poly_degree, px, py, pz);
    int N = k + np;
    int nops = dim == 3 ? 4 : 3;
    /* rows are independent: each OpenMP thread solves its rows with its own scratch */
#pragma omp parallel
    {
    double *A = (double *)malloc(sizeof(double) * (size_t)N * N);
    double *Ai = (double *)malloc(sizeof(double) * (size_t)N * N);
    double *aug = (double *)malloc(sizeof(double) * (size_t)N * 2 * N);
    double **rows = (double **)malloc(sizeof(double *) * (size_t)N);
    double *L = (double *)malloc(sizeof(double) * (size_t)N);
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < n; i++) {
        const int *cl = cloud + (size_t)i * k;
        build_A(k, np, dim, phs, cl, x, y, z, px, py, pz, A);
        gauss_jordan(N, A, Ai, aug, rows);
        for (int o = 0; o < nops; o++) {
            int op = (o == nops - 1) ? 3 : o;
            double *D = op == 0 ? Dx : op == 1 ? Dy : op == 2 ? Dz : lap;
            operator_row0(op, k, np, dim, phs, cl, x, y, z, px, py, pz, L);
            for (int j = 0; j < k; j++) {
                double s = 0;
                for (int c = 0; c < N; c++) s += L[c] * Ai[(size_t)c * N + j];
                D[(size_t)i * k + j] = s;
            }
        }
        for (int j = 0; j < k; j++) {
            size_t o = (size_t)i * k + j;
            if (btag[i]) {
                double v = Dx[o] * nx[i] + Dy[o] * ny[i];
                if (dim == 3) v += Dz[o] * nz[i];
                lapP[o] = v;
            } else lapP[o] = lap[o];
        }
    }
    free(A); free(Ai); free(aug); free(rows); free(L);
    }
}

/* create_restriction_matrix / create_prolongation_matrix (mesh_functions.h:533-670):
 * interpolation weights from the source level's cloud around src_pt[i] to target
 * node i.  rows_from: first target row computed (the reference starts at
 * num_boundary_nodes, :563/:633; rows before it stay 0).  If only_interior,
 * rows with a boundary tag are skipped instead (the convergent solver's variant). */
ORC_EXPORT void orc_transfer_weights(int nt, const double *tx, const double *ty, const double *tz,
                                     const unsigned char *tbtag, const int *src_pt, int rows_from, int only_interior,
                                     int ns, int ks, int dim, int phs, int poly_degree_src,
                                     const double *sx, const double *sy, const double *sz, const int *scloud,
                                     double *W /* [nt][ks] */)
{
    (void)ns;
    short px[64], py[64], pz[64];
    int np = orc_monomials(dim, poly_degree_src, px, py, pz);
    int m = ks, N = ks + np;
    memset(W, 0, sizeof(double) * (size_t)nt * ks);
    /* rows are independent: each OpenMP thread solves its rows with its own scratch */
#pragma omp parallel
    {
    double *A = (double *)malloc(sizeof(double) * (size_t)N * N);
    double *Ai = (double *)malloc(sizeof(double) * (size_t)N * N);
    double *aug = (double *)malloc(sizeof(double) * (size_t)N * 2 * N);
    double **rows = (double **)malloc(sizeof(double *) * (size_t)N);
    double *tmp = (double *)malloc(sizeof(double) * (size_t)N);
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < nt; i++) {
        if (only_interior ? (tbtag[i] != 0) : (i < rows_from)) continue;
        int ip = src_pt[i];
        const int *cl = scloud + (size_t)ip * ks;
        build_A(m, np, dim, phs, cl, sx, sy, sz, px, py, pz, A);
        gauss_jordan(N, A, Ai, aug, rows);
        double p1[3] = {tx[i], ty[i], tz[i]};
        for (int j = 0; j < m; j++) {
            double p2[3] = {sx[cl[j]], sy[cl[j]], sz[cl[j]]};
            tmp[j] = phs_rbf(p1, p2, phs, dim);
        }
        double seed[3] = {sx[ip], sy[ip], sz[ip]};
        for (int j = 0; j < np; j++)
            tmp[j + m] = pow(p1[0] - seed[0], px[j]) * pow(p1[1] - seed[1], py[j]) * pow(p1[2] - seed[2], pz[j]);
        for (int c = 0; c < m; c++) {
            double s = 0;
            for (int j = 0; j < N; j++) s += tmp[j] * Ai[(size_t)j * N + c];
            W[(size_t)i * ks + c] = s;
        }
    }
    free(A); free(Ai); free(aug); free(rows); free(tmp);
    }
}

/* ------------------------------------------------------------------------ */
/* Stencil operations of fractional_step_solver.h / mat_lib.h               */
/* ------------------------------------------------------------------------ */

/* multiply_sparse_matrix_vector_gpu (mat_lib.h:80-89) */
ORC_EXPORT void orc_spmv(int n, int k, const double *D, const int *cloud, const double *f, double *out)
{
    for (int i = 0; i < n; i++) {
        double r = 0.0;
        for (int j = 0; j < k; j++) r += D[(size_t)i * k + j] * f[cloud[(size_t)i * k + j]];
        out[i] = r;
    }
}

/* Level-0 state of the fractional step (FieldVariables members it touches). */
typedef struct {
    double *u, *v, *w, *p, *u_new, *v_new, *w_new, *u_old, *v_old, *w_old;
    double *res, *source, *dpdn, *dpdx, *dpdy, *dpdz;
} orc_field;

typedef struct {
    int n, k, dim;
    const int *cloud;
    const unsigned char *btag;
    const double *x, *y, *z;   /* set by orc_ctx_coords (the heat program's sources need them) */
    const double *nx, *ny, *nz;
    const double *Dx, *Dy, *Dz, *lap, *lapP;
    /* transfer data of this level */
    const int *rpts, *ppts;
    const double *restr; /* [n][k_finer] */
    const double *prol;  /* [n][k_coarser] */
} orc_level;

/* calculate_intermediate_velocity (fractional_step_solver.h:73-114) */
static void intermediate_velocity(const orc_level *L, orc_field *f, double dt, double nu)
{
    int n = L->n, k = L->k;
    double *vel[3] = {f->u, f->v, f->w};
    double *out[3] = {f->u_new, f->v_new, f->w_new};
    int ncomp = L->dim == 3 ? 3 : 2;
    for (int c = 0; c < ncomp; c++) {
        orc_spmv(n, k, L->Dx, L->cloud, vel[c], f->dpdx);
        orc_spmv(n, k, L->Dy, L->cloud, vel[c], f->dpdy);
        if (L->dim == 3) orc_spmv(n, k, L->Dz, L->cloud, vel[c], f->dpdz);
        orc_spmv(n, k, L->lap, L->cloud, vel[c], f->dpdn);
        for (int i = 0; i < n; i++)
            out[c][i] = vel[c][i] - dt * (f->u[i] * f->dpdx[i] + f->v[i] * f->dpdy[i] + f->w[i] * f->dpdz[i] - nu * f->dpdn[i]);
    }
}

/* calculate_mass_residual (fractional_step_solver.h:116-131) */
static void mass_residual(const orc_level *L, orc_field *f, double dt, double rho)
{
    int n = L->n, k = L->k;
    orc_spmv(n, k, L->Dx, L->cloud, f->u_new, f->dpdx);
    orc_spmv(n, k, L->Dy, L->cloud, f->v_new, f->dpdy);
    if (L->dim == 3) orc_spmv(n, k, L->Dz, L->cloud, f->w_new, f->dpdz);
    for (int i = 0; i < n; i++)
        if (!L->btag[i]) f->source[i] = rho * (f->dpdx[i] + f->dpdy[i] + f->dpdz[i]) / dt;
}

/* calculate_boundary_dpdn (fractional_step_solver.h:133-148) */
static void boundary_dpdn(const orc_level *L, orc_field *f, double dt, double rho)
{
    for (int i = 0; i < L->n; i++) {
        if (!L->btag[i]) continue;
        double dx = (f->u_new[i] - f->u[i]) * rho / dt;
        double dy = (f->v_new[i] - f->v[i]) * rho / dt;
        f->dpdn[i] = dx * L->nx[i] + dy * L->ny[i];
        if (L->dim == 3) {
            double dz = (f->w_new[i] - f->w[i]) * rho / dt;
            f->dpdn[i] += dz * L->nz[i];
        }
    }
}

/* relaxation (fractional_step_solver.h:168-196).  jacobi = 0: the in-place
 * sweep of the C build (Gauss-Seidel order); jacobi = 1: every node updated
 * from the previous sweep's values (the data-parallel order the GPU uses). */
static void relaxation(const orc_level *L, double *p, const double *source, double *res,
                       float omega, int num_relax, int jacobi, double *scratch)
{
    int n = L->n, k = L->k;
    double w1 = omega, w2 = (1 - omega);
    for (int it = 0; it < num_relax; it++) {
        const double *pin = p;
        if (jacobi) { memcpy(scratch, p, sizeof(double) * (size_t)n); pin = scratch; }
        for (int i = 0; i < n; i++) {
            double sum = 0.0;
            for (int j = 1; j < k; j++) sum += L->lapP[(size_t)i * k + j] * pin[L->cloud[(size_t)i * k + j]];
            p[i] = w1 * ((source[i] - sum) / L->lapP[(size_t)i * k]) + w2 * pin[i];
        }
        double pref = p[0];
        for (int i = 0; i < n; i++) p[i] = p[i] - pref;
        for (int i = 0; i < n; i++) {
            res[i] = source[i];
            for (int j = 0; j < k; j++) res[i] = res[i] - L->lap[(size_t)i * k + j] * p[L->cloud[(size_t)i * k + j]];
        }
    }
}

/* calculate_residuals (fractional_step_solver.h:236-246) */
static void residuals_interior(const orc_level *L, const double *p, const double *source, double *res)
{
    int n = L->n, k = L->k;
    for (int i = 0; i < n; i++) {
        if (L->btag[i]) continue;
        double sum = 0;
        for (int j = 0; j < k; j++) sum += L->lap[(size_t)i * k + j] * p[L->cloud[(size_t)i * k + j]];
        res[i] = source[i] - sum;
    }
}

/* restrict_residuals (fractional_step_solver.h:198-212) */
static void restrict_res(const orc_level *F, const orc_level *C, const double *res_f, double *source_c)
{
    for (int i = 0; i < C->n; i++) {
        if (C->btag[i]) continue;
        double r = 0.0;
        int ir = C->rpts[i];
        for (int j = 0; j < F->k; j++) r += C->restr[(size_t)i * F->k + j] * res_f[F->cloud[(size_t)ir * F->k + j]];
        source_c[i] = r;
    }
}

/* prolongate_corrections (fractional_step_solver.h:214-234) */
static void prolongate(const orc_level *F, const orc_level *C, double *p_f, double *p_c)
{
    for (int i = 0; i < F->n; i++) {
        if (F->btag[i]) continue;
        int ip = F->ppts[i];
        double r = 0.0;
        for (int j = 0; j < C->k; j++) r += F->prol[(size_t)i * C->k + j] * p_c[C->cloud[(size_t)ip * C->k + j]];
        p_f[i] = p_f[i] + r;
    }
    for (int i = 0; i < C->n; i++) if (!C->btag[i]) p_c[i] = 0.0;
}

/* multigrid_Poisson_solver (fractional_step_solver.h:150-166), on per-level
 * arrays p[l], source[l], res[l]. */
static void multigrid(int nl, const orc_level *Ls, double **p, double **source, double **res,
                      float omega, int num_relax, int num_vcycles, int jacobi, double *scratch)
{
    for (int cyc = 0; cyc < num_vcycles; cyc++) {
        for (int l = 0; l < nl; l++) {
            relaxation(&Ls[l], p[l], source[l], res[l], omega, num_relax, jacobi, scratch);
            residuals_interior(&Ls[l], p[l], source[l], res[l]);
            if (l != nl - 1) restrict_res(&Ls[l], &Ls[l + 1], res[l], source[l + 1]);
        }
        for (int l = nl - 1; l > 0; l--) {
            prolongate(&Ls[l - 1], &Ls[l], p[l - 1], p[l]);
            if (l != 1) relaxation(&Ls[l - 1], p[l - 1], source[l - 1], res[l - 1], omega, num_relax, jacobi, scratch);
        }
    }
}

/* update_velocity (fractional_step_solver.h:248-275); returns the printed mass residual. */
static double update_velocity(const orc_level *L, orc_field *f, double dt, double rho)
{
    int n = L->n, k = L->k;
    orc_spmv(n, k, L->Dx, L->cloud, f->p, f->dpdx);
    orc_spmv(n, k, L->Dy, L->cloud, f->p, f->dpdy);
    if (L->dim == 3) orc_spmv(n, k, L->Dz, L->cloud, f->p, f->dpdz);
    for (int i = 0; i < n; i++) {
        if (L->btag[i]) continue;
        f->u[i] = f->u_new[i] - dt * f->dpdx[i] / rho;
        f->v[i] = f->v_new[i] - dt * f->dpdy[i] / rho;
        if (L->dim == 3) f->w[i] = f->w_new[i] - dt * f->dpdz[i] / rho;
    }
    orc_spmv(n, k, L->Dx, L->cloud, f->u, f->dpdx);
    orc_spmv(n, k, L->Dy, L->cloud, f->v, f->dpdy);
    double s = 0.0;
    for (int i = 0; i < n; i++) s += rho * fabs(f->dpdx[i] + f->dpdy[i]);
    return s / n;
}

/* ---- flat entry points for the tests (ctypes) --------------------------- */

#define MAXL 16
typedef struct {
    int nl, dim;
    orc_level L[MAXL];
    double *p[MAXL], *source[MAXL], *res[MAXL];
    orc_field f;
    double dt, nu, rho;
    float omega;
    int num_relax, num_vcycles, jacobi;
    double *scratch;
} orc_ctx;

ORC_EXPORT void *orc_ctx_new(int nl, int dim) { orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx)); c->nl = nl; c->dim = dim; return c; }
ORC_EXPORT void orc_ctx_free(void *h) { orc_ctx *c = (orc_ctx *)h; free(c->scratch); free(c); }

/* All arrays are borrowed (owned by the caller, kept alive for the handle's life). */
ORC_EXPORT void orc_ctx_level(void *h, int l, int n, int k, const int *cloud, const unsigned char *btag,
                              const double *nx, const double *ny, const double *nz,
                              const double *Dx, const double *Dy, const double *Dz, const double *lap, const double *lapP,
                              const int *rpts, const int *ppts, const double *restr, const double *prol,
                              double *p, double *source, double *res)
{
    orc_ctx *c = (orc_ctx *)h;
    orc_level *L = &c->L[l];
    L->n = n; L->k = k; L->dim = c->dim; L->cloud = cloud; L->btag = btag;
    L->nx = nx; L->ny = ny; L->nz = nz;
    L->Dx = Dx; L->Dy = Dy; L->Dz = Dz; L->lap = lap; L->lapP = lapP;
    L->rpts = rpts; L->ppts = ppts; L->restr = restr; L->prol = prol;
    c->p[l] = p; c->source[l] = source; c->res[l] = res;
    if (l == 0) {
        free(c->scratch);
        c->scratch = (double *)malloc(sizeof(double) * (size_t)n);
    }
}

/* fields: u v w u_new v_new w_new u_old v_old w_old dpdn dpdx dpdy dpdz (level 0) */
ORC_EXPORT void orc_ctx_fields(void *h, double *u, double *v, double *w, double *u_new, double *v_new, double *w_new,
                               double *u_old, double *v_old, double *w_old, double *dpdn, double *dpdx, double *dpdy, double *dpdz)
{
    orc_ctx *c = (orc_ctx *)h;
    orc_field *f = &c->f;
    f->u = u; f->v = v; f->w = w; f->u_new = u_new; f->v_new = v_new; f->w_new = w_new;
    f->u_old = u_old; f->v_old = v_old; f->w_old = w_old; f->dpdn = dpdn; f->dpdx = dpdx; f->dpdy = dpdy; f->dpdz = dpdz;
    f->p = c->p[0]; f->source = c->source[0]; f->res = c->res[0];
}

ORC_EXPORT void orc_ctx_params(void *h, double dt, double Re, float omega, int num_relax, int num_vcycles, int jacobi)
{
    orc_ctx *c = (orc_ctx *)h;
    c->rho = 1; c->nu = (c->rho / Re) / c->rho; c->dt = dt; c->omega = omega;
    c->num_relax = num_relax; c->num_vcycles = num_vcycles; c->jacobi = jacobi;
}

ORC_EXPORT void orc_multigrid(void *h)
{
    orc_ctx *c = (orc_ctx *)h;
    multigrid(c->nl, c->L, c->p, c->source, c->res, c->omega, c->num_relax, c->num_vcycles, c->jacobi, c->scratch);
}

ORC_EXPORT void orc_relaxation(void *h, int l)
{
    orc_ctx *c = (orc_ctx *)h;
    relaxation(&c->L[l], c->p[l], c->source[l], c->res[l], c->omega, c->num_relax, c->jacobi, c->scratch);
}

/* fractional_step_explicit (fractional_step_solver.h:47-71); mass residual of
 * update_velocity returned through *mass_res when non-NULL. */
ORC_EXPORT double orc_step(void *h, double *mass_res)
{
    orc_ctx *c = (orc_ctx *)h;
    orc_level *L = &c->L[0];
    orc_field *f = &c->f;
    int n = L->n;
    for (int i = 0; i < n; i++) { f->u_old[i] = f->u[i]; f->v_old[i] = f->v[i]; if (c->dim == 3) f->w_old[i] = f->w[i]; }
    intermediate_velocity(L, f, c->dt, c->nu);
    mass_residual(L, f, c->dt, c->rho);
    boundary_dpdn(L, f, c->dt, c->rho);
    multigrid(c->nl, c->L, c->p, c->source, c->res, c->omega, c->num_relax, c->num_vcycles, c->jacobi, c->scratch);
    double mr = update_velocity(L, f, c->dt, c->rho);
    if (mass_res) *mass_res = mr;
    double e = 0.0;
    for (int i = 0; i < n; i++) {
        e += (f->u[i] - f->u_old[i]) * (f->u[i] - f->u_old[i]) + (f->v[i] - f->v_old[i]) * (f->v[i] - f->v_old[i]);
        if (c->dim == 3) e += (f->w[i] - f->w_old[i]) * (f->w[i] - f->w_old[i]);
    }
    return sqrt(e / n);
}

ORC_EXPORT void orc_intermediate_velocity(void *h) { orc_ctx *c = (orc_ctx *)h; intermediate_velocity(&c->L[0], &c->f, c->dt, c->nu); }
ORC_EXPORT void orc_mass_residual(void *h) { orc_ctx *c = (orc_ctx *)h; mass_residual(&c->L[0], &c->f, c->dt, c->rho); }
ORC_EXPORT double orc_update_velocity(void *h) { orc_ctx *c = (orc_ctx *)h; return update_velocity(&c->L[0], &c->f, c->dt, c->rho); }

/* ------------------------------------------------------------------------ */
/* TIMPLE: the time-implicit step (timple_solver.h:40-410), the default      */
/* solver of mg_NS_solver.c.  Per level p[l] holds pprime; p_old is level 0. */
/* jacobi = 0: the in-place sweeps of the C build; jacobi = 1: every node   */
/* updated from the previous sweep's values (the GPU's order).              */
/* ------------------------------------------------------------------------ */
typedef struct {
    double *p_old;
    int iter_timple, iter_momentum;
    double facRe, facdt;
    const int *color;   /* jacobi == 2: the momentum sweeps' colours (orc_ctx_timple_colors) */
    int ncolors;
    double *su, *sv, *sw;  /* previous-sweep copies (Jacobi order) */
} orc_timple;

static orc_timple g_timple;

/* the colours of the momentum sweeps in colour order (jacobi == 2); borrowed */
ORC_EXPORT void orc_ctx_timple_colors(void *h, const int *color, int ncolors)
{
    orc_ctx *c = (orc_ctx *)h;
    c->jacobi = 2;
    g_timple.color = color;
    g_timple.ncolors = ncolors;
}

ORC_EXPORT void orc_ctx_timple(void *h, double *p_old, int iter_timple, int iter_momentum, double facRe, double facdt)
{
    orc_ctx *c = (orc_ctx *)h;
    int n = c->L[0].n;
    g_timple.p_old = p_old;
    g_timple.iter_timple = iter_timple;
    g_timple.iter_momentum = iter_momentum;
    g_timple.facRe = facRe;
    g_timple.facdt = facdt;
    free(g_timple.su); free(g_timple.sv); free(g_timple.sw);
    g_timple.su = (double *)malloc(sizeof(double) * (size_t)n);
    g_timple.sv = (double *)malloc(sizeof(double) * (size_t)n);
    g_timple.sw = (double *)malloc(sizeof(double) * (size_t)n);
}

/* calculate_intermediate_velocity_implicit (timple_solver.h:72-175) */
static void timple_momentum(orc_ctx *c)
{
    const orc_level *L = &c->L[0];
    orc_field *f = &c->f;
    const orc_timple *t = &g_timple;
    int n = L->n, k = L->k, dim = c->dim;
    /* mu = rho / Re; with rho = 1 (mesh_functions.h:97) this is nu * rho, bit for bit */
    double rho = c->rho, mu = c->nu * c->rho, dt = c->dt;
    orc_spmv(n, k, L->Dx, L->cloud, t->p_old, f->dpdx);
    orc_spmv(n, k, L->Dy, L->cloud, t->p_old, f->dpdy);
    if (dim == 3) orc_spmv(n, k, L->Dz, L->cloud, t->p_old, f->dpdz);
    for (int it = 0; it < t->iter_momentum; it++) {
        const double *uin = f->u_new, *vin = f->v_new, *win = f->w_new;
        if (c->jacobi == 1) {
            memcpy(t->su, f->u_new, sizeof(double) * (size_t)n); uin = t->su;
            memcpy(t->sv, f->v_new, sizeof(double) * (size_t)n); vin = t->sv;
            if (dim == 3) { memcpy(t->sw, f->w_new, sizeof(double) * (size_t)n); win = t->sw; }
        }
        /* jacobi == 2: in place, colour by colour (no two nodes of a colour in
         * each other's clouds, so a colour's nodes may go in any order) */
        const int passes = c->jacobi == 2 ? t->ncolors : 1;
        for (int pass = 0; pass < passes; pass++)
        for (int i = 0; i < n; i++) {
            if (L->btag[i]) continue;
            if (c->jacobi == 2 && t->color[i] != pass) continue;
            const size_t r = (size_t)i * k;
            const double *comp_in[3] = {uin, vin, win};
            double *comp_out[3] = {f->u_new, f->v_new, f->w_new};
            const double *comp_old[3] = {f->u_old, f->v_old, f->w_old};
            const double *grad[3] = {f->dpdx, f->dpdy, f->dpdz};
            for (int cidx = 0; cidx < (dim == 3 ? 3 : 2); cidx++) {
                const double *x = comp_in[cidx];
                double temp1 = 0, temp2 = 0, temp3 = 0, temp4 = 0;
                double advection_x = f->u[i] * L->Dx[r];
                double advection_y = f->v[i] * L->Dy[r];
                double diffusion = -t->facRe * mu * L->lap[r];
                double unsteady = 1. / (dt * t->facdt);
                double denom;
                if (cidx < 2) {
                    denom = rho * (advection_x + advection_y + unsteady) + diffusion;
                    for (int j = 1; j < k; j++) {
                        double xv = x[L->cloud[r + j]];
                        temp1 += L->Dx[r + j] * xv;
                        temp2 += L->Dy[r + j] * xv;
                        temp4 += L->lap[r + j] * xv;
                    }
                    if (dim == 3) {
                        denom += rho * f->w[i] * L->Dz[r];
                        for (int j = 1; j < k; j++) temp3 += L->Dz[r + j] * x[L->cloud[r + j]];
                    }
                } else {
                    double advection_z = f->w[i] * L->Dz[r];
                    denom = rho * (advection_x + advection_y + advection_z + unsteady) + diffusion;
                    for (int j = 1; j < k; j++) {
                        double xv = x[L->cloud[r + j]];
                        temp1 += L->Dx[r + j] * xv;
                        temp2 += L->Dy[r + j] * xv;
                        temp3 += L->Dz[r + j] * xv;
                        temp4 += L->lap[r + j] * xv;
                    }
                }
                double advection = f->u[i] * temp1 + f->v[i] * temp2 + f->w[i] * temp3;
                unsteady = comp_old[cidx][i] / (dt * t->facdt);
                comp_out[cidx][i] = (rho * (unsteady - advection) - (t->facRe - 1) * mu * L->lap[r] * x[i] +
                                     mu * temp4 - grad[cidx][i]) / denom;
            }
        }
    }
}

/* calculate_mass_residual_implicit (timple_solver.h:177-201) */
static void timple_mass(orc_ctx *c)
{
    const orc_level *L = &c->L[0];
    orc_field *f = &c->f;
    int n = L->n, k = L->k;
    orc_spmv(n, k, L->Dx, L->cloud, f->u_new, f->dpdx);
    orc_spmv(n, k, L->Dy, L->cloud, f->v_new, f->dpdy);
    if (c->dim == 3) orc_spmv(n, k, L->Dz, L->cloud, f->w_new, f->dpdz);
    for (int i = 0; i < n; i++)
        f->source[i] = L->btag[i] ? 0 : c->rho * (f->dpdx[i] + f->dpdy[i] + f->dpdz[i]) / c->dt;
}

/* relaxation (timple_solver.h:249-283): residual with lap_Poison on interior rows */
static void timple_relaxation(const orc_level *L, double *p, const double *source, double *res, float omega,
                              int num_relax, int jacobi, double *scratch)
{
    int n = L->n, k = L->k;
    for (int it = 0; it < num_relax; it++) {
        const double *pin = p;
        if (jacobi) { memcpy(scratch, p, sizeof(double) * (size_t)n); pin = scratch; }
        for (int i = 0; i < n; i++) {
            double sum = 0.0;
            for (int j = 1; j < k; j++) sum += L->lapP[(size_t)i * k + j] * pin[L->cloud[(size_t)i * k + j]];
            p[i] = omega * ((source[i] - sum) / L->lapP[(size_t)i * k]) + (1 - omega) * pin[i];
        }
        double pref = p[0];
        for (int i = 0; i < n; i++) p[i] = p[i] - pref;
        for (int i = 0; i < n; i++) {
            if (!L->btag[i]) {
                res[i] = source[i];
                for (int j = 0; j < k; j++) res[i] = res[i] - L->lapP[(size_t)i * k + j] * p[L->cloud[(size_t)i * k + j]];
            } else res[i] = 0;
        }
    }
}

/* calculate_residuals (timple_solver.h:285-301) */
static void timple_residuals(const orc_level *L, const double *p, const double *source, double *res)
{
    int n = L->n, k = L->k;
    for (int i = 0; i < n; i++) {
        res[i] = 0.0;
        if (!L->btag[i]) {
            double sum = 0;
            for (int j = 0; j < k; j++) sum += L->lapP[(size_t)i * k + j] * p[L->cloud[(size_t)i * k + j]];
            res[i] = source[i] - sum;
        }
    }
}

/* restrict_residuals (timple_solver.h:303-317): every coarse row written */
static void timple_restrict(const orc_level *F, const orc_level *C, const double *res_f, double *source_c)
{
    for (int i = 0; i < C->n; i++) {
        double results = 0.0;
        if (!C->btag[i]) {
            int ir = C->rpts[i];
            for (int j = 0; j < F->k; j++) results += C->restr[(size_t)i * F->k + j] * res_f[F->cloud[(size_t)ir * F->k + j]];
        }
        source_c[i] = results;
    }
}

/* prolongate_corrections (timple_solver.h:319-339): every coarse pprime reset */
static void timple_prolongate(const orc_level *F, const orc_level *C, double *p_f, double *p_c)
{
    for (int i = 0; i < F->n; i++) {
        if (F->btag[i]) continue;
        int ip = F->ppts[i];
        double r = 0.0;
        for (int j = 0; j < C->k; j++) r += F->prol[(size_t)i * C->k + j] * p_c[C->cloud[(size_t)ip * C->k + j]];
        p_f[i] = p_f[i] + r;
    }
    for (int i = 0; i < C->n; i++) p_c[i] = 0.0;
}

/* multigrid_Poisson_solver (timple_solver.h:203-220) */
static void timple_multigrid(orc_ctx *c)
{
    int nl = c->nl;
    for (int cyc = 0; cyc < c->num_vcycles; cyc++) {
        for (int l = 0; l < nl; l++) {
            timple_relaxation(&c->L[l], c->p[l], c->source[l], c->res[l], c->omega, c->num_relax, c->jacobi, c->scratch);
            timple_residuals(&c->L[l], c->p[l], c->source[l], c->res[l]);
            if (l != nl - 1) timple_restrict(&c->L[l], &c->L[l + 1], c->res[l], c->source[l + 1]);
        }
        for (int l = nl - 1; l > 0; l--) {
            timple_prolongate(&c->L[l - 1], &c->L[l], c->p[l - 1], c->p[l]);
            if (l != 1)
                timple_relaxation(&c->L[l - 1], c->p[l - 1], c->source[l - 1], c->res[l - 1], c->omega, c->num_relax,
                                  c->jacobi, c->scratch);
        }
    }
}

/* update_velocity_implicit (timple_solver.h:341-369) */
static void timple_update_velocity(orc_ctx *c)
{
    const orc_level *L = &c->L[0];
    orc_field *f = &c->f;
    int n = L->n, k = L->k;
    double *pp = c->p[0], *p_old = g_timple.p_old;
    orc_spmv(n, k, L->Dx, L->cloud, pp, f->dpdx);
    orc_spmv(n, k, L->Dy, L->cloud, pp, f->dpdy);
    if (c->dim == 3) orc_spmv(n, k, L->Dz, L->cloud, pp, f->dpdz);
    for (int i = 0; i < n; i++) {
        if (L->btag[i]) continue;
        f->u_new[i] = f->u_new[i] - c->dt * f->dpdx[i] / c->rho;
        f->v_new[i] = f->v_new[i] - c->dt * f->dpdy[i] / c->rho;
        if (c->dim == 3) f->w_new[i] = f->w_new[i] - c->dt * f->dpdz[i] / c->rho;
        p_old[i] = p_old[i] + 1.0 * pp[i];
    }
    double pref = p_old[0];
    for (int i = 0; i < n; i++) p_old[i] = p_old[i] - pref;
}

/* update_boundary_pressure (timple_solver.h:371-410).  The velocity terms are
 * assigned, not accumulated, inside the stencil loop (:378-380), so only the
 * last stencil slot contributes; FieldVariables.rho, which the reference never
 * sets, is taken as rho. */
static void timple_boundary_pressure(orc_ctx *c)
{
    const orc_level *L = &c->L[0];
    orc_field *f = &c->f;
    int n = L->n, k = L->k, dim = c->dim;
    double *p_old = g_timple.p_old;
    double nu = c->nu;
    for (int i = 0; i < n; i++) {
        if (!L->btag[i]) continue;
        const size_t r = (size_t)i * k;
        double temp1 = 0, temp2 = 0, temp3 = 0;
        for (int j = 0; j < k; j++) {
            int cj = L->cloud[r + j];
            temp1 = nu * L->lap[r + j] * f->u_new[cj];
            temp1 -= f->u[i] * f->u_new[cj] * L->Dx[r + j];
            temp1 -= f->v[i] * f->u_new[cj] * L->Dy[r + j];
            if (dim == 3) temp1 -= f->w[i] * f->u_new[cj] * L->Dz[r + j];
            temp2 = nu * L->lap[r + j] * f->v_new[cj];
            temp2 -= f->u[i] * f->v_new[cj] * L->Dx[r + j];
            temp2 -= f->v[i] * f->v_new[cj] * L->Dy[r + j];
            if (dim == 3) temp2 -= f->w[i] * f->v_new[cj] * L->Dz[r + j];
            if (dim == 3) {
                temp3 = nu * L->lap[r + j] * f->w_new[cj];
                temp3 -= f->u[i] * f->w_new[cj] * L->Dx[r + j];
                temp3 -= f->v[i] * f->w_new[cj] * L->Dy[r + j];
                temp3 -= f->w[i] * f->w_new[cj] * L->Dz[r + j];
            }
        }
        f->dpdn[i] = c->rho * (temp1 * L->nx[i] + temp2 * L->ny[i] + temp3 * L->nz[i]);
        double sumx = 0, sumy = 0, sumz = 0, Ap = 0.0;
        for (int j = 1; j < k; j++) {
            sumx += L->Dx[r + j] * p_old[L->cloud[r + j]];
            sumy += L->Dy[r + j] * p_old[L->cloud[r + j]];
            if (dim == 3) sumz += L->Dz[r + j] * p_old[L->cloud[r + j]];
        }
        Ap += L->Dx[r] * L->nx[i];
        Ap += L->Dy[r] * L->ny[i];
        if (dim == 3) Ap += L->Dz[r] * L->nz[i];
        p_old[i] = (f->dpdn[i] - sumx * L->nx[i] - sumy * L->ny[i] - sumz * L->nz[i]) / Ap;
    }
}

/* time_implicit_solver (timple_solver.h:40-70) */
ORC_EXPORT double orc_timple_step(void *h)
{
    orc_ctx *c = (orc_ctx *)h;
    orc_field *f = &c->f;
    int n = c->L[0].n, dim = c->dim;
    double *pp = c->p[0];
    for (int i = 0; i < n; i++) {
        f->u_old[i] = f->u_new[i]; f->u[i] = f->u_new[i];
        f->v_old[i] = f->v_new[i]; f->v[i] = f->v_new[i];
        f->w_old[i] = f->w_new[i]; f->w[i] = f->w_new[i];
        pp[i] = 0;
    }
    for (int it = 0; it < g_timple.iter_timple; it++) {
        for (int i = 0; i < n; i++) { f->u[i] = f->u_new[i]; f->v[i] = f->v_new[i]; f->w[i] = f->w_new[i]; pp[i] = 0; }
        timple_momentum(c);
        timple_mass(c);
        timple_multigrid(c);
        timple_update_velocity(c);
        timple_boundary_pressure(c);
    }
    double e = 0.0;
    for (int i = 0; i < n; i++) {
        e += pow(f->u_new[i] - f->u_old[i], 2) + pow(f->v_new[i] - f->v_old[i], 2);
        if (dim == 3) e += pow(f->w_new[i] - f->w_old[i], 2);
    }
    return sqrt(e / n);
}

ORC_EXPORT void orc_timple_momentum(void *h) { timple_momentum((orc_ctx *)h); }
ORC_EXPORT void orc_timple_mass(void *h) { timple_mass((orc_ctx *)h); }
ORC_EXPORT void orc_timple_multigrid(void *h) { timple_multigrid((orc_ctx *)h); }
ORC_EXPORT void orc_timple_update_velocity(void *h) { timple_update_velocity((orc_ctx *)h); }
ORC_EXPORT void orc_timple_boundary_pressure(void *h) { timple_boundary_pressure((orc_ctx *)h); }

/* ------------------------------------------------------------------------ */
/* read_PointStructure (mesh_functions.h:172-476): Gmsh 2.2 ASCII reader.   */
/* Nodes from $Nodes; boundary tags and unnormalised normals from the       */
/* boundary elements (2D: 2-node lines, normal (-dy, dx) added to both      */
/* nodes; 3D: 3-node triangles and 4-node quads, the cross product of the   */
/* element's first two edges from node 1 added to every node), corner tags  */
/* from 1-node points (and, in 3D, from both ends of 2-node lines); every   */
/* element line holds three integers between its type and its nodes.  The   */
/* first num_corners nodes are then dropped (Gmsh numbers the geometric     */
/* points first).  d_avg = sqrt(Lx Ly / num_elem) in 2D, cbrt(Lx Ly Lz /    */
/* num_elem) in 3D over the bounding box, min/max started at +-1e6.         */
/* Returns the node count after the removal (-1: unreadable file); with     */
/* cap >= that count the arrays are filled too.                             */
/* ------------------------------------------------------------------------ */
static int gm_seek(FILE *f, const char *word)
{
    char tok[64];
    for (;;) {
        if (fscanf(f, "%63s ", tok) != 1) return -1;
        if (strcmp(tok, word) == 0) return 0;
    }
}

ORC_EXPORT int orc_read_gmsh(const char *path, int dim, int cap, double *x, double *y, double *z,
                             double *nx, double *ny, double *nz, unsigned char *btag, unsigned char *corner,
                             int *nb, int *num_elem, double *d_avg)
{
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    int nn = 0, ne = 0, id = 0;
    if (gm_seek(f, "$Nodes") || fscanf(f, "%i ", &nn) != 1 || nn <= 0) { fclose(f); return -1; }
    double *X = calloc((size_t)nn, sizeof(double)), *Y = calloc((size_t)nn, sizeof(double));
    double *Z = calloc((size_t)nn, sizeof(double)), *NX = calloc((size_t)nn, sizeof(double));
    double *NY = calloc((size_t)nn, sizeof(double)), *NZ = calloc((size_t)nn, sizeof(double));
    unsigned char *BT = calloc((size_t)nn, 1), *CT = calloc((size_t)nn, 1);
    double lo[3] = {1e6, 1e6, 1e6}, hi[3] = {-1e6, -1e6, -1e6};
    int ok = 1;
    for (int i = 0; i < nn && ok; i++) {
        double v[3];
        ok = fscanf(f, "%i ", &id) == 1 && fscanf(f, "%lf ", &v[0]) == 1 && fscanf(f, "%lf ", &v[1]) == 1 &&
             fscanf(f, "%lf ", &v[2]) == 1;
        X[i] = v[0]; Y[i] = v[1]; Z[i] = v[2];
        for (int d = 0; d < 3; d++) {
            if (v[d] < lo[d]) lo[d] = v[d];
            if (v[d] > hi[d]) hi[d] = v[d];
        }
    }
    if (ok) ok = gm_seek(f, "$Elements") == 0 && fscanf(f, "%i ", &ne) == 1;
    for (int e = 0; e < ne && ok; e++) {
        int type = 0, t[3], a = 0, b = 0, c = 0, q = 0;
        ok = fscanf(f, "%i ", &id) == 1 && fscanf(f, "%i ", &type) == 1;
        if (!ok) break;
        const int two_d_line = dim == 2 && type == 1, tri = dim == 3 && type == 2, quad = dim == 3 && type == 3;
        const int line3 = dim == 3 && type == 1, point = type == 15;
        if (!(two_d_line || tri || quad || line3 || point)) {
            if (fscanf(f, "%*[^\n]\n") == EOF) ok = 0;
            continue;
        }
        ok = fscanf(f, "%i ", &t[0]) == 1 && fscanf(f, "%i ", &t[1]) == 1 && fscanf(f, "%i ", &t[2]) == 1;
        if (!ok) break;
        if (point) {
            ok = fscanf(f, "%i ", &a) == 1 && a >= 1 && a <= nn;
            if (ok) CT[a - 1] = 1;
        } else if (line3) {
            ok = fscanf(f, "%i ", &a) == 1 && fscanf(f, "%i ", &b) == 1 && a >= 1 && a <= nn && b >= 1 && b <= nn;
            if (ok) { CT[a - 1] = 1; CT[b - 1] = 1; }
        } else if (two_d_line) {
            ok = fscanf(f, "%i ", &a) == 1 && fscanf(f, "%i ", &b) == 1 && a >= 1 && a <= nn && b >= 1 && b <= nn;
            if (!ok) break;
            a--; b--;
            BT[a] = 1; BT[b] = 1;
            const double dx = X[b] - X[a], dy = Y[b] - Y[a];
            NX[a] += -dy; NY[a] += dx;
            NX[b] += -dy; NY[b] += dx;
        } else {
            ok = fscanf(f, "%i ", &a) == 1 && fscanf(f, "%i ", &b) == 1 && fscanf(f, "%i ", &c) == 1 &&
                 a >= 1 && a <= nn && b >= 1 && b <= nn && c >= 1 && c <= nn;
            if (ok && quad) ok = fscanf(f, "%i ", &q) == 1 && q >= 1 && q <= nn;
            if (!ok) break;
            int nodes[4] = {a - 1, b - 1, c - 1, quad ? q - 1 : -1};
            const int cnt = quad ? 4 : 3;
            for (int m = 0; m < cnt; m++) BT[nodes[m]] = 1;
            const int A = nodes[0], B = nodes[1], C = nodes[2];
            const double dx = X[B] - X[A], dy = Y[B] - Y[A], dz = Z[B] - Z[A];
            const double dx1 = X[C] - X[A], dy1 = Y[C] - Y[A], dz1 = Z[C] - Z[A];
            const double cx = dy * dz1 - dz * dy1, cy = dz * dx1 - dx * dz1, cz = dx * dy1 - dy * dx1;
            for (int m = 0; m < cnt; m++) NX[nodes[m]] += cx;
            for (int m = 0; m < cnt; m++) NY[nodes[m]] += cy;
            for (int m = 0; m < cnt; m++) NZ[nodes[m]] += cz;
        }
    }
    fclose(f);
    int n = -1;
    if (ok) {
        int nbnd = 0, ncorner = 0;
        for (int i = 0; i < nn; i++) { nbnd += BT[i] != 0; ncorner += CT[i] != 0; }
        n = nn - ncorner;
        if (num_elem) *num_elem = ne;
        if (nb) *nb = nbnd - ncorner;
        if (d_avg) {
            const double L0 = hi[0] - lo[0], L1 = hi[1] - lo[1], L2 = hi[2] - lo[2];
            *d_avg = dim == 2 ? sqrt(L0 * L1 / ne) : cbrt(L0 * L1 * L2 / ne);
        }
        if (cap >= n) {
            for (int i = 0; i < n; i++) {
                const int s = i + ncorner;
                x[i] = X[s]; y[i] = Y[s]; z[i] = Z[s];
                nx[i] = NX[s]; ny[i] = NY[s]; nz[i] = NZ[s];
                btag[i] = BT[s]; corner[i] = CT[s];
            }
        }
    }
    free(X); free(Y); free(Z); free(NX); free(NY); free(NZ); free(BT); free(CT);
    return n;
}

/* ------------------------------------------------------------------------ */
/* The heat-conduction program (mg_heat_conduction.c:43-83 with             */
/* heat_conduction.h:24-113 and init/init_heat_conduction.c:14-67): a      */
/* manufactured Poisson problem with Dirichlet rows (boundary nodes at      */
/* x == 0) and Neumann rows (the other boundary nodes) solved by the       */
/* program's own V-cycle.  jacobi = 0: in-place sweeps (the C build);      */
/* jacobi = 1: every node from the previous sweep's values (the GPU).      */
/* ------------------------------------------------------------------------ */
ORC_EXPORT void orc_ctx_coords(void *h, int l, const double *x, const double *y, const double *z)
{
    orc_ctx *c = (orc_ctx *)h;
    c->L[l].x = x; c->L[l].y = y; c->L[l].z = z;
}

/* relaxation (heat_conduction.h:24-48): SOR over every row with lap_Poison,
 * nothing else (no re-pin, no residual) */
static void heat_relaxation(const orc_level *L, double *p, const double *source, float omega, int num_relax,
                            int jacobi, double *scratch)
{
    int n = L->n, k = L->k;
    for (int it = 0; it < num_relax; it++) {
        const double *pin = p;
        if (jacobi) { memcpy(scratch, p, sizeof(double) * (size_t)n); pin = scratch; }
        for (int i = 0; i < n; i++) {
            double sum = 0.0;
            for (int j = 1; j < k; j++) sum += L->lapP[(size_t)i * k + j] * pin[L->cloud[(size_t)i * k + j]];
            p[i] = omega * ((source[i] - sum) / L->lapP[(size_t)i * k]) + (1 - omega) * pin[i];
        }
    }
}

/* calculate_residuals (heat_conduction.h:100-113): lap_Poison, boundary rows 0 */
static void heat_residuals(const orc_level *L, const double *p, const double *source, double *res)
{
    int n = L->n, k = L->k;
    for (int i = 0; i < n; i++) {
        res[i] = 0.0;
        if (L->btag[i]) continue;
        double sum = 0;
        for (int j = 0; j < k; j++) sum += L->lapP[(size_t)i * k + j] * p[L->cloud[(size_t)i * k + j]];
        res[i] = source[i] - sum;
    }
}

/* restrict_residuals (heat_conduction.h:50-69): every coarse row written, boundary rows 0 */
static void heat_restrict(const orc_level *F, const orc_level *C, const double *res_f, double *source_c)
{
    for (int i = 0; i < C->n; i++) {
        double r = 0.0;
        if (!C->btag[i]) {
            int ir = C->rpts[i];
            for (int j = 0; j < F->k; j++) r += C->restr[(size_t)i * F->k + j] * res_f[F->cloud[(size_t)ir * F->k + j]];
        }
        source_c[i] = r;
    }
}

/* the cycle of mg_heat_conduction.c:58-71 (prolongate_corrections,
 * heat_conduction.h:71-98, is the fractional step's) */
static void heat_cycle(orc_ctx *c)
{
    const int nl = c->nl;
    for (int l = 0; l < nl; l++) {
        heat_relaxation(&c->L[l], c->p[l], c->source[l], c->omega, c->num_relax, c->jacobi, c->scratch);
        heat_residuals(&c->L[l], c->p[l], c->source[l], c->res[l]);
        if (l != nl - 1) heat_restrict(&c->L[l], &c->L[l + 1], c->res[l], c->source[l + 1]);
    }
    for (int l = nl - 1; l > 0; l--) {
        prolongate(&c->L[l - 1], &c->L[l], c->p[l - 1], c->p[l]);
        if (l != 1) heat_relaxation(&c->L[l - 1], c->p[l - 1], c->source[l - 1], c->omega, c->num_relax, c->jacobi,
                                    c->scratch);
    }
}

/* initial_conditions + boundary_conditions (init_heat_conduction.c:14-49):
 * res = p = 0 everywhere, level-0 source -8 pi^2 k^2 sin(2 pi k x) sin(2 pi k y)
 * with pi written 3.14, coarse sources 0 */
ORC_EXPORT void orc_heat_init(void *h, int wave)
{
    orc_ctx *c = (orc_ctx *)h;
    const int k = wave;
    for (int l = 0; l < c->nl; l++) {
        const orc_level *L = &c->L[l];
        for (int i = 0; i < L->n; i++) {
            c->res[l][i] = 0.0;
            c->source[l][i] = l == 0 ? -8 * 3.14 * 3.14 * k * k * sin(2 * 3.14 * k * c->L[0].x[i]) *
                                           sin(2 * 3.14 * k * c->L[0].y[i])
                                     : 0.0;
            c->p[l][i] = 0.0;
        }
    }
}

/* set_boundary_rhs (init_heat_conduction.c:51-65), level 0: boundary nodes at
 * x == 0 become Dirichlet rows (lap_Poison row = e_i, source 1), the others
 * get the manufactured solution's normal derivative as their source */
ORC_EXPORT void orc_heat_boundary_rhs(void *h, int wave)
{
    orc_ctx *c = (orc_ctx *)h;
    orc_level *L = &c->L[0];
    const int k = wave, kk = L->k;
    double *lapP = (double *)L->lapP;
    for (int i = 0; i < L->n; i++) {
        if (!L->btag[i]) continue;
        const double x = L->x[i], y = L->y[i];
        if (x == 0) {
            c->source[0][i] = 1.0;
            for (int j = 0; j < kk; j++) lapP[(size_t)i * kk + j] = 0.0;
            lapP[(size_t)i * kk] = 1.0;
        } else {
            c->source[0][i] = 2 * 3.14 * k * (sin(2 * 3.14 * k * x) * cos(2 * 3.14 * k * y) * L->ny[i] +
                                              cos(2 * 3.14 * k * x) * sin(2 * 3.14 * k * y) * L->nx[i]);
        }
    }
}

/* one time step of mg_heat_conduction.c:47-77: num_vcycles cycles, each after
 * set_boundary_rhs; returns the sum over level 0 of (p_before - p_after)^2 */
ORC_EXPORT double orc_heat_step(void *h, int wave)
{
    orc_ctx *c = (orc_ctx *)h;
    const int n = c->L[0].n;
    double *temp = (double *)malloc(sizeof(double) * (size_t)n);
    memcpy(temp, c->p[0], sizeof(double) * (size_t)n);
    for (int cyc = 0; cyc < c->num_vcycles; cyc++) {
        orc_heat_boundary_rhs(h, wave);
        heat_cycle(c);
    }
    double e = 0.0;
    for (int i = 0; i < n; i++) e += (temp[i] - c->p[0][i]) * (temp[i] - c->p[0][i]);
    free(temp);
    return e;
}

/* matrixInverse_Gauss_Jordan (mat_lib.h:423-491) of one row-major N x N matrix */
ORC_EXPORT void orc_gauss_jordan(int N, const double *A, double *Ainv)
{
    double *aug = (double *)malloc(sizeof(double) * (size_t)N * 2 * N);
    double **rows = (double **)malloc(sizeof(double *) * (size_t)N);
    gauss_jordan(N, A, Ainv, aug, rows);
    free(aug);
    free(rows);
}
