// weights.cuh -- device routines of the per-node saddle-point weight solve,
// shared by the fixed-stencil kernels (setup.cu) and the persistent
// uneven-size batch (batch_setup.cu).
//
// One system of order N = m + np (m stencil nodes, np monomials) is solved by
// a Team: a whole CTA, or a slice of it synchronised by a named barrier.  The
// arithmetic is that of the reference: create_A_matrix_from_cloud_indices
// (rbf.h:42-77), the operator rows of gradx/grady/gradz/laplacian_matrix
// (rbf.h:79-270) and matrixInverse_Gauss_Jordan (mat_lib.h:423-491: a single
// bubble pass on column 0, no further pivoting), with every product and
// difference rounded separately.  Which thread computes an element does not
// change its value.
#pragma once
#include "mgm_internal.cuh"

namespace mgm {

struct MonoDev {
    int np;
    short px[kMaxPoly], py[kMaxPoly], pz[kMaxPoly];
};

inline MonoDev to_dev(const Monomials &m)
{
    MonoDev d;
    d.np = m.np;
    for (int i = 0; i < kMaxPoly; i++) { d.px[i] = m.px[i]; d.py[i] = m.py[i]; d.pz[i] = m.pz[i]; }
    return d;
}

// A group of `size` consecutive threads of a CTA (tid: the thread's rank in it).
// bar 0: the whole CTA (__syncthreads); otherwise named barrier `bar`.
struct Team {
    int tid, size, bar;
    __device__ static Team block() { return Team{(int)threadIdx.x, (int)blockDim.x, 0}; }
    __device__ void sync() const
    {
        if (bar == 0) __syncthreads();
        else if (size == 32) __syncwarp();
        else asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(size) : "memory");
    }
};

// Shared-memory doubles one system needs: aug[N][2N] | sx,sy,sz[m] | L[4][N] | t[N] | out[4][m], then perm[N] ints.
__host__ __device__ inline size_t system_doubles(int m, int np)
{
    const int N = m + np;
    return (size_t)N * 2 * N + 3 * (size_t)m + 4 * (size_t)N + N + 4 * (size_t)m;
}
__host__ __device__ inline size_t system_bytes(int m, int np)
{
    // rounded up to 16 bytes so that consecutive slots stay aligned
    return ((sizeof(double) * system_doubles(m, np) + sizeof(int) * (size_t)(m + np)) + 15) & ~(size_t)15;
}

__device__ __forceinline__ void stage_cloud(const Team &tm, const int *cl, int m, const double *x, const double *y,
                                            const double *z, double *sx, double *sy, double *sz)
{
    for (int j = tm.tid; j < m; j += tm.size) { int c = cl[j]; sx[j] = x[c]; sy[j] = y[c]; sz[j] = z[c]; }
}

// create_A_matrix_from_cloud_indices (rbf.h:42-77) into the left half of aug,
// identity into the right half.
__device__ inline void build_aug(const Team &tm, int m, int np, int dim, int phs, const MonoDev &mono,
                                 const double *sx, const double *sy, const double *sz, double *aug, int N)
{
    const int W2 = 2 * N;
    for (int e = tm.tid; e < N * W2; e += tm.size) {
        int i = e / W2, j = e % W2;
        double v;
        if (j >= N) v = (j - N == i) ? 1.0 : 0.0;
        else if (i < m && j < m) {
            if (i == j) v = 0;
            else {
                int a = min(i, j), b = max(i, j);  // the reference evaluates (cloud[a], cloud[b]) with a < b
                double p1[3] = {sx[a], sy[a], sz[a]}, p2[3] = {sx[b], sy[b], sz[b]};
                v = mgm_phs_rbf(p1, p2, phs, dim);
            }
        } else if (i < m || j < m) {
            int node = i < m ? i : j, t = i < m ? j - m : i - m;
            v = 1;
            if (mono.px[t] != 0) v = MGM_MUL(v, mgm_pow_int(MGM_SUB(sx[node], sx[0]), mono.px[t]));
            if (mono.py[t] != 0) v = MGM_MUL(v, mgm_pow_int(MGM_SUB(sy[node], sy[0]), mono.py[t]));
            if (mono.pz[t] != 0) v = MGM_MUL(v, mgm_pow_int(MGM_SUB(sz[node], sz[0]), mono.pz[t]));
        } else v = 0;
        aug[e] = v;
    }
}

// In-place Gauss-Jordan; on return aug[perm[i]][N + j] holds inverse[i][j].
// Elimination by column ownership: a thread keeps the pivot-row entry of its
// column in a register and sweeps the rows (all of them, or every R-th row when
// the team has R >= 2 threads per column).
__device__ inline void gauss_jordan(const Team &tm, double *aug, int *perm, double *t, int N)
{
    const int W2 = 2 * N;
    if (tm.tid == 0) {
        for (int i = 0; i < N; i++) perm[i] = i;
        for (int i = N - 1; i > 0; i--)
            if (aug[perm[i - 1] * W2] < aug[perm[i] * W2]) { int tmp = perm[i]; perm[i] = perm[i - 1]; perm[i - 1] = tmp; }
    }
    tm.sync();
    for (int i = 0; i < N; i++) {
        const double *pr = aug + perm[i] * W2;
        const double piv = pr[i];
        for (int j = tm.tid; j < N; j += tm.size) t[j] = (j == i) ? 0.0 : MGM_DIV(aug[perm[j] * W2 + i], piv);
        tm.sync();
        if (tm.size >= 2 * W2) {
            // enough threads for several row groups per column
            const int R = tm.size / W2;
            if (tm.tid < R * W2) {
                const int c = tm.tid % W2;
                const double pc = pr[c];
                for (int j = tm.tid / W2; j < N; j += R) {
                    if (j == i) continue;
                    double *rj = aug + perm[j] * W2;
                    rj[c] = MGM_SUB(rj[c], MGM_MUL(pc, t[j]));
                }
            }
        } else {
            for (int c = tm.tid; c < W2; c += tm.size) {
                const double pc = pr[c];
                for (int j = 0; j < N; j++) {
                    if (j == i) continue;
                    double *rj = aug + perm[j] * W2;
                    rj[c] = MGM_SUB(rj[c], MGM_MUL(pc, t[j]));
                }
            }
        }
        tm.sync();
    }
    for (int e = tm.tid; e < N * N; e += tm.size) {
        int i = e / N, j = e % N;
        double *ri = aug + perm[i] * W2;
        ri[N + j] = MGM_DIV(ri[N + j], ri[i]);
    }
    tm.sync();
}

// Row 0 of gradx/grady/gradz/laplacian_matrix (rbf.h:79-270) at the seed.
// op: 0 d/dx, 1 d/dy, 2 d/dz, 3 Laplacian.
__device__ inline void operator_row0(const Team &tm, int op, int m, int np, int dim, int phs, const MonoDev &mono,
                                     const double *sx, const double *sy, const double *sz, double *L)
{
    const int N = m + np;
    const double p1[3] = {sx[0], sy[0], sz[0]};
    for (int c = tm.tid; c < N; c += tm.size) {
        double v = 0;
        if (c < m) {
            const double p2[3] = {sx[c], sy[c], sz[c]};
            if (op <= 2) v = MGM_MUL(MGM_MUL((double)phs, MGM_SUB(p1[op], p2[op])), mgm_phs_rbf(p1, p2, phs - 2, dim));
            else v = MGM_MUL((double)(phs * phs), mgm_phs_rbf(p1, p2, phs - 2, dim));
            if ((op == 1 || op == 2) && c == 0) v = 0;  // rbf.h:141, :180 zero column 0
        } else {
            const int j = c - m;
            const double d0 = MGM_SUB(p1[0], sx[0]), d1 = MGM_SUB(p1[1], sy[0]), d2 = MGM_SUB(p1[2], sz[0]);
            const int ex = mono.px[j], ey = mono.py[j], ez = mono.pz[j];
            if (op == 0) {
                if (j == 0 || ex == 0) v = 0;
                else { v = MGM_MUL((double)ex, mgm_pow_int(d0, ex - 1)); v = MGM_MUL(v, mgm_pow_int(d1, ey)); v = MGM_MUL(v, mgm_pow_int(d2, ez)); }
            } else if (op == 1) {
                if (j == 0 || ey == 0) v = 0;  // grad[i][m] is never written by grady_matrix: zero from create_matrix
                else { v = MGM_MUL((double)ey, mgm_pow_int(d1, ey - 1)); v = MGM_MUL(v, mgm_pow_int(d0, ex)); v = MGM_MUL(v, mgm_pow_int(d2, ez)); }
            } else if (op == 2) {
                if (j == 0 || ez == 0) v = 0;
                else { v = MGM_MUL((double)ez, mgm_pow_int(d2, ez - 1)); v = MGM_MUL(v, mgm_pow_int(d1, ey)); v = MGM_MUL(v, mgm_pow_int(d0, ex)); }
            } else {
                double tx = 0, ty = 0, tz = 0;
                if (ex > 1) {
                    tx = MGM_MUL((double)(ex * (ex - 1)), mgm_pow_int(d0, ex - 2));
                    tx = MGM_MUL(tx, mgm_pow_int(d1, ey));
                    if (dim == 3) tx = MGM_MUL(tx, mgm_pow_int(d2, ez));
                } else if (ey > 1) {
                    ty = MGM_MUL((double)(ey * (ey - 1)), mgm_pow_int(d1, ey - 2));
                    ty = MGM_MUL(ty, mgm_pow_int(d0, ex));
                    if (dim == 3) ty = MGM_MUL(ty, mgm_pow_int(d2, ez));
                } else if (dim == 3 && ez > 1) {
                    tz = MGM_MUL((double)(ez * (ez - 1)), mgm_pow_int(d2, ez - 2));
                    tz = MGM_MUL(tz, mgm_pow_int(d0, ex));
                    tz = MGM_MUL(tz, mgm_pow_int(d1, ey));
                }
                v = dim == 3 ? MGM_ADD(MGM_ADD(tx, ty), tz) : MGM_ADD(tx, ty);
            }
        }
        L[c] = v;
    }
}

// Interpolation row of create_restriction/prolongation_matrix (mesh_functions.h:533-670):
// the PHS and monomials of the target point p1 relative to the source seed.
__device__ inline void transfer_row(const Team &tm, int m, int np, int dim, int phs, const MonoDev &mono,
                                    const double *sx, const double *sy, const double *sz, const double p1[3],
                                    const double seed[3], double *tmp)
{
    const int N = m + np;
    for (int c = tm.tid; c < N; c += tm.size) {
        double v;
        if (c < m) {
            const double p2[3] = {sx[c], sy[c], sz[c]};
            v = mgm_phs_rbf(p1, p2, phs, dim);
        } else {
            const int j = c - m;
            v = MGM_MUL(MGM_MUL(mgm_pow_int(MGM_SUB(p1[0], seed[0]), mono.px[j]),
                                mgm_pow_int(MGM_SUB(p1[1], seed[1]), mono.py[j])),
                        mgm_pow_int(MGM_SUB(p1[2], seed[2]), mono.pz[j]));
        }
        tmp[c] = v;
    }
}

// out[j] = sum_c row[c] * inverse[c][j], c ascending (multiply_matrices, mat_lib.h:214-228,
// and multiply_vector_matrix_columnwise, mat_lib.h:720-726), for j < m.
__device__ __forceinline__ double row_times_inverse(const double *row, const double *aug, const int *perm, int N, int j)
{
    double s = 0;
    for (int c = 0; c < N; c++) s = MGM_ADD(s, MGM_MUL(row[c], aug[perm[c] * 2 * N + N + j]));
    return s;
}

}  // namespace mgm
