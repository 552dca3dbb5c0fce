// batch_solve.cu -- B right-hand sides through one V-cycle hierarchy.
//
// The system and preconditioner are those of the single-RHS solve (solver.cu):
// the pinned operator (lap_Poison with row 0 replaced by p[0] = 0), Chebyshev
// smoothing in D^-1 A on interior rows with an exact solve of the boundary rows
// after every step, restriction of the interior residual, prolongation shifted
// so that the pinned node gets no correction, a dense coarsest inverse, and
// flexible GMRES in FP64 outside.  Every vector is node-major [n][B]: a warp
// owns a row, its lanes own Q = B/32 consecutive right-hand sides, so a
// stencil weight and index are loaded once for all B right-hand sides and
// every gathered neighbour is one contiguous B-wide access.
#include <algorithm>
#include <cmath>

#include "batch.cuh"

namespace mgm {

constexpr int kBatchMaxRestart = 32;

template <class T, int Q>
__device__ __forceinline__ void ldq(const T *p, T (&v)[Q])
{
    if constexpr (Q == 2) {
        if constexpr (sizeof(T) == 4) { const float2 t = *(const float2 *)p; v[0] = t.x; v[1] = t.y; }
        else { const double2 t = *(const double2 *)p; v[0] = t.x; v[1] = t.y; }
    } else v[0] = *p;
}
template <class T, int Q>
__device__ __forceinline__ void ldgq(const T *p, T (&v)[Q])
{
    if constexpr (Q == 2) {
        if constexpr (sizeof(T) == 4) { const float2 t = __ldg((const float2 *)p); v[0] = t.x; v[1] = t.y; }
        else { const double2 t = __ldg((const double2 *)p); v[0] = t.x; v[1] = t.y; }
    } else v[0] = __ldg(p);
}
template <class T, int Q>
__device__ __forceinline__ void stq(T *p, const T (&v)[Q])
{
    if constexpr (Q == 2) {
        if constexpr (sizeof(T) == 4) *(float2 *)p = make_float2(v[0], v[1]);
        else *(double2 *)p = make_double2(v[0], v[1]);
    } else *p = v[0];
}

// acc[q] = sum_j A[beg + j] * x[col[beg + j]][lane*Q + q], j ascending.  The
// row's indices and weights are loaded by the lanes 32 at a time and
// broadcast; eight gathers are in flight per warp.
template <class T, int Q, class X>
__device__ __forceinline__ void row_dot_b(const int *__restrict__ col, const T *__restrict__ A, int beg, int cnt,
                                          const X *__restrict__ x, int B, int lane, T (&acc)[Q])
{
#pragma unroll
    for (int q = 0; q < Q; q++) acc[q] = T(0);
    for (int j0 = 0; j0 < cnt; j0 += 32) {
        const int jj = j0 + lane;
        int c = 0;
        T a = T(0);
        if (jj < cnt) { c = __ldg(col + beg + jj); a = __ldg(A + beg + jj); }
        const int m = min(32, cnt - j0);
        int t = 0;
        for (; t + 8 <= m; t += 8) {
            int cc[8];
            T aa[8];
            X xv[8][Q];
#pragma unroll
            for (int u = 0; u < 8; u++) { cc[u] = __shfl_sync(0xffffffffu, c, t + u); aa[u] = __shfl_sync(0xffffffffu, a, t + u); }
#pragma unroll
            for (int u = 0; u < 8; u++) ldgq<X, Q>(x + (long)cc[u] * B + lane * Q, xv[u]);
#pragma unroll
            for (int u = 0; u < 8; u++)
#pragma unroll
                for (int q = 0; q < Q; q++) acc[q] += aa[u] * (T)xv[u][q];
        }
        for (; t < m; t++) {
            const int ct = __shfl_sync(0xffffffffu, c, t);
            const T at = __shfl_sync(0xffffffffu, a, t);
            X xv[Q];
            ldgq<X, Q>(x + (long)ct * B + lane * Q, xv);
#pragma unroll
            for (int q = 0; q < Q; q++) acc[q] += at * (T)xv[q];
        }
    }
}

// Row-kernel shape: a CTA of 8 warps owns kRowsPerCta consecutive rows and
// its warps step through them together (warp w: rows w, w + 8, ...).  In the
// breadth-first order consecutive rows share most neighbours, so the gathered
// neighbour rows of one CTA are served from L1 after their first use.
constexpr int kRowsPerCta = 64;
inline int rows_grid(long rows) { return blocks_for(rows, kRowsPerCta); }
#define MGM_CTA_ROWS(r, count)                                                                     \
    for (int r##_k = (int)(threadIdx.x >> 5), r = blockIdx.x * kRowsPerCta + r##_k;                \
         r##_k < kRowsPerCta && r < (count); r##_k += 8, r += 8)

// exact solve of the boundary rows (they couple only to themselves and interior nodes)
template <class T, int Q>
__global__ void __launch_bounds__(256) k_b_bnd(int nbl, const int *__restrict__ list, const int *__restrict__ rp,
                                               const int *__restrict__ col, const T *__restrict__ A,
                                               const T *__restrict__ dinv, const T *__restrict__ r, T *e, int B,
                                               int zero_start)
{
    const int lane = threadIdx.x & 31;
    MGM_CTA_ROWS(w, nbl) {
        const int i = list[w];
        const long o = (long)i * B + lane * Q;
        T rv[Q], ev[Q];
        ldq<T, Q>(r + o, rv);
        const T di = dinv[i];
        if (zero_start) {
#pragma unroll
            for (int q = 0; q < Q; q++) ev[q] = rv[q] * di;
        } else {
            T acc[Q];
            row_dot_b<T, Q, T>(col, A, rp[i], rp[i + 1] - rp[i], e, B, lane, acc);
            ldq<T, Q>(e + o, ev);
#pragma unroll
            for (int q = 0; q < Q; q++) ev[q] = ev[q] + (rv[q] - acc[q]) * di;
        }
        stq<T, Q>(e + o, ev);
    }
}

// one Chebyshev step on interior rows: q = r - A e, d = c1 d + c2 D^-1 q, e' = e + d
template <class T, int Q>
__global__ void __launch_bounds__(256) k_b_cheb(int n, const int *__restrict__ rp, const int *__restrict__ col,
                                                const T *__restrict__ A, const T *__restrict__ dinv,
                                                const uint8_t *__restrict__ btag, const T *__restrict__ r,
                                                const T *__restrict__ e, T *__restrict__ eout, T *__restrict__ d,
                                                int B, T c1, T c2, int first)
{
    const int lane = threadIdx.x & 31;
    MGM_CTA_ROWS(i, n) {
        const long o = (long)i * B + lane * Q;
        T ev[Q];
        ldq<T, Q>(e + o, ev);
        if (btag[i]) { stq<T, Q>(eout + o, ev); continue; }
        T acc[Q], rv[Q], dv[Q];
        row_dot_b<T, Q, T>(col, A, rp[i], rp[i + 1] - rp[i], e, B, lane, acc);
        ldq<T, Q>(r + o, rv);
        if (!first) ldq<T, Q>(d + o, dv);
        const T di = dinv[i];
#pragma unroll
        for (int q = 0; q < Q; q++) {
            const T qv = rv[q] - acc[q];
            dv[q] = first ? c2 * di * qv : c1 * dv[q] + c2 * di * qv;
            ev[q] += dv[q];
        }
        stq<T, Q>(d + o, dv);
        stq<T, Q>(eout + o, ev);
    }
}

template <class T, int Q>
__global__ void __launch_bounds__(256) k_b_residual(int n, const int *__restrict__ rp, const int *__restrict__ col,
                                                    const T *__restrict__ A, const uint8_t *__restrict__ btag,
                                                    const T *__restrict__ r, const T *__restrict__ e,
                                                    T *__restrict__ qo, int B)
{
    const int lane = threadIdx.x & 31;
    MGM_CTA_ROWS(i, n) {
        const long o = (long)i * B + lane * Q;
        T out[Q];
        if (btag[i]) {
#pragma unroll
            for (int q = 0; q < Q; q++) out[q] = T(0);
        } else {
            T acc[Q], rv[Q];
            row_dot_b<T, Q, T>(col, A, rp[i], rp[i + 1] - rp[i], e, B, lane, acc);
            ldq<T, Q>(r + o, rv);
#pragma unroll
            for (int q = 0; q < Q; q++) out[q] = rv[q] - acc[q];
        }
        stq<T, Q>(qo + o, out);
    }
}

// y = M x for a CSR transfer matrix (empty rows give 0)
template <class T, int Q>
__global__ void __launch_bounds__(256) k_b_restrict(int n, const int *__restrict__ rp, const int *__restrict__ col,
                                                    const T *__restrict__ w, const T *__restrict__ x,
                                                    T *__restrict__ y, int B)
{
    const int lane = threadIdx.x & 31;
    MGM_CTA_ROWS(i, n) {
        T acc[Q];
        row_dot_b<T, Q, T>(col, w, rp[i], rp[i + 1] - rp[i], x, B, lane, acc);
        stq<T, Q>(y + (long)i * B + lane * Q, acc);
    }
}

// ef += P ec - (P ec)[row 0]
template <class T, int Q>
__global__ void __launch_bounds__(256) k_b_prolong(int n, const int *__restrict__ rp, const int *__restrict__ col,
                                                   const T *__restrict__ w, const T *__restrict__ ec,
                                                   T *__restrict__ ef, int B)
{
    __shared__ T shift[64];
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < 32) {
        T acc[Q];
        row_dot_b<T, Q, T>(col, w, rp[0], rp[1] - rp[0], ec, B, lane, acc);
#pragma unroll
        for (int q = 0; q < Q; q++) shift[lane * Q + q] = acc[q];
    }
    __syncthreads();
    MGM_CTA_ROWS(i, n) {
        T acc[Q], ev[Q];
        row_dot_b<T, Q, T>(col, w, rp[i], rp[i + 1] - rp[i], ec, B, lane, acc);
        const long o = (long)i * B + lane * Q;
        ldq<T, Q>(ef + o, ev);
#pragma unroll
        for (int q = 0; q < Q; q++) ev[q] += acc[q] - shift[lane * Q + q];
        stq<T, Q>(ef + o, ev);
    }
}

// E[n][B] = inv[n][n] R[n][B]; block: 32 rows x B columns, K tiles of 32
template <class T, int B>
__global__ void __launch_bounds__(256) k_b_dense(int n, const T *__restrict__ inv, const T *__restrict__ R,
                                                 T *__restrict__ E)
{
    constexpr int RPT = B / 8;  // rows per thread
    __shared__ T a[32][33];
    __shared__ T rt[32][B];
    const int tid = threadIdx.x, b = tid % B, rg = tid / B;
    const int row0 = blockIdx.x * 32;
    T acc[RPT];
#pragma unroll
    for (int u = 0; u < RPT; u++) acc[u] = T(0);
    for (int k0 = 0; k0 < n; k0 += 32) {
        for (int e = tid; e < 32 * 32; e += 256) {
            const int rr = e / 32, kk = e % 32;
            a[rr][kk] = (row0 + rr < n && k0 + kk < n) ? inv[(long)(row0 + rr) * n + k0 + kk] : T(0);
        }
        for (int e = tid; e < 32 * B; e += 256) {
            const int kk = e / B, bb = e % B;
            rt[kk][bb] = k0 + kk < n ? R[(long)(k0 + kk) * B + bb] : T(0);
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < 32; kk++) {
            const T rv = rt[kk][b];
#pragma unroll
            for (int u = 0; u < RPT; u++) acc[u] += a[rg * RPT + u][kk] * rv;
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < RPT; u++) {
        const int row = row0 + rg * RPT + u;
        if (row < n) E[(long)row * B + b] = acc[u];
    }
}

// ---------------------------------------------------------------------------
// FP64 Krylov kernels on [n][B] vectors
// ---------------------------------------------------------------------------
// r = b - A x, per-block partial |r_b|^2 and |b_b|^2: part[(blk*2 + {0,1})*B + b]
template <class X, int Q>
__global__ void __launch_bounds__(256) k_b_resid64(int n, const int *__restrict__ rp, const int *__restrict__ col,
                                                   const double *__restrict__ A, const double *__restrict__ bv,
                                                   const X *__restrict__ x, double *__restrict__ r,
                                                   double *__restrict__ part, int B)
{
    __shared__ double srr[8][64], sbb[8][64];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double rr[Q], bb[Q];
#pragma unroll
    for (int q = 0; q < Q; q++) rr[q] = bb[q] = 0.0;
    for (int i = blockIdx.x * 8 + wib; i < n; i += gridDim.x * 8) {
        double acc[Q], bq[Q];
        row_dot_b<double, Q, X>(col, A, rp[i], rp[i + 1] - rp[i], x, B, lane, acc);
        const long o = (long)i * B + lane * Q;
        ldq<double, Q>(bv + o, bq);
#pragma unroll
        for (int q = 0; q < Q; q++) { acc[q] = bq[q] - acc[q]; rr[q] += acc[q] * acc[q]; bb[q] += bq[q] * bq[q]; }
        stq<double, Q>(r + o, acc);
    }
#pragma unroll
    for (int q = 0; q < Q; q++) { srr[wib][lane * Q + q] = rr[q]; sbb[wib][lane * Q + q] = bb[q]; }
    __syncthreads();
    if (threadIdx.x < B) {
        double a = 0, c = 0;
        for (int w = 0; w < 8; w++) { a += srr[w][threadIdx.x]; c += sbb[w][threadIdx.x]; }
        part[((long)blockIdx.x * 2 + 0) * B + threadIdx.x] = a;
        part[((long)blockIdx.x * 2 + 1) * B + threadIdx.x] = c;
    }
}

template <class X, int Q>
__global__ void __launch_bounds__(256) k_b_apply64(int n, const int *__restrict__ rp, const int *__restrict__ col,
                                                   const double *__restrict__ A, const X *__restrict__ z,
                                                   double *__restrict__ w, int B)
{
    const int lane = threadIdx.x & 31;
    MGM_CTA_ROWS(i, n) {
        double acc[Q];
        row_dot_b<double, Q, X>(col, A, rp[i], rp[i + 1] - rp[i], z, B, lane, acc);
        stq<double, Q>(w + (long)i * B + lane * Q, acc);
    }
}

// part[(blk*cnt + c)*B + b] = sum over this block's rows of V_c[i][b] W[i][b]
__global__ void __launch_bounds__(256) k_b_multidot(int n, int B, int cnt, const double *__restrict__ V, long ldv,
                                                    const double *__restrict__ W, double *__restrict__ part)
{
    __shared__ double sm[8][256];
    const int b = threadIdx.x % B, rs = threadIdx.x / B, R = 256 / B;
    for (int c0 = 0; c0 < cnt; c0 += 8) {
        const int cc = min(8, cnt - c0);
        double acc[8];
#pragma unroll
        for (int u = 0; u < 8; u++) acc[u] = 0.0;
        for (long i = (long)blockIdx.x * R + rs; i < n; i += (long)gridDim.x * R) {
            const double wv = W[i * B + b];
#pragma unroll
            for (int u = 0; u < 8; u++)
                if (u < cc) acc[u] = fma(V[(c0 + u) * ldv + i * B + b], wv, acc[u]);
        }
#pragma unroll
        for (int u = 0; u < 8; u++) sm[u][threadIdx.x] = acc[u];
        __syncthreads();
        if (threadIdx.x < B) {
            for (int u = 0; u < cc; u++) {
                double s = 0;
                for (int q = 0; q < R; q++) s += sm[u][q * B + threadIdx.x];
                part[((long)blockIdx.x * cnt + c0 + u) * B + threadIdx.x] = s;
            }
        }
        __syncthreads();
    }
}

// out[c*B + b] = sum_blk part[(blk*cnt + c)*B + b]; one CTA per (c, 32 columns),
// 8 warps summing interleaved blocks, then a fixed-order sum of the 8 partials.
__global__ void __launch_bounds__(256) k_b_reduce(const double *__restrict__ part, int nblk, int cnt, int B,
                                                  double *__restrict__ out)
{
    __shared__ double sm[8][33];
    const int chunks = (B + 31) / 32;
    const int c = blockIdx.x / chunks, b = (blockIdx.x % chunks) * 32 + (threadIdx.x & 31), w = threadIdx.x >> 5;
    double s = 0;
    if (b < B)
        for (int k = w; k < nblk; k += 8) s += part[((long)k * cnt + c) * B + b];
    sm[w][threadIdx.x & 31] = s;
    __syncthreads();
    if (w == 0 && b < B) {
        double t = 0;
        for (int q = 0; q < 8; q++) t += sm[q][threadIdx.x];
        out[c * B + b] = t;
    }
}

// W -= sum_c h[c][b] V_c, and per-block partial |W_b|^2 of the result:
// part[blk*B + b].  Grid-stride over elements; the stride is a multiple of B,
// so a thread keeps one right-hand side.
__global__ void __launch_bounds__(256) k_b_orth_norm(long nB, int B, int cnt, const double *__restrict__ V, long ldv,
                                                     const double *__restrict__ h, double *__restrict__ W,
                                                     double *__restrict__ part)
{
    __shared__ double hs[kBatchMaxRestart + 1][64];
    __shared__ double sq[256];
    for (int t = threadIdx.x; t < cnt * B; t += blockDim.x) hs[t / B][t % B] = h[t];
    __syncthreads();
    const int b = threadIdx.x % B;
    double acc = 0.0;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < nB; e += (long)gridDim.x * blockDim.x) {
        double s = W[e];
        for (int c = 0; c < cnt; c++) s = fma(-hs[c][b], V[c * ldv + e], s);
        W[e] = s;
        acc = fma(s, s, acc);
    }
    sq[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < B) {
        double a = 0;
        for (int q = threadIdx.x; q < (int)blockDim.x; q += B) a += sq[q];
        part[(long)blockIdx.x * B + threadIdx.x] = a;
    }
}

// out = in / nrm_b  (nrm holds |.|^2 when is_sq)
__global__ void k_b_scale(long nB, int B, const double *__restrict__ in, double *__restrict__ out,
                          const double *__restrict__ nrm, int is_sq)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nB) return;
    const double v = nrm[e % B];
    const double d = is_sq ? sqrt(v) : v;
    out[e] = d > 0 ? in[e] / d : 0.0;
}

// X += sum_c y[c][b] Z_c
template <class T>
__global__ void __launch_bounds__(256) k_b_combine(long nB, int B, int cnt, const T *__restrict__ Z, long ldz,
                                                   const double *__restrict__ y, double *__restrict__ X)
{
    __shared__ double ys[kBatchMaxRestart + 1][64];
    for (int t = threadIdx.x; t < cnt * B; t += blockDim.x) ys[t / B][t % B] = y[t];
    __syncthreads();
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nB) return;
    const int b = (int)(e % B);
    double s = X[e];
    for (int c = 0; c < cnt; c++) s = fma(ys[c][b], (double)Z[c * ldz + e], s);
    X[e] = s;
}

template <class T, class U>
__global__ void k_b_convert(long nB, const T *__restrict__ in, U *__restrict__ out)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nB) out[e] = (U)in[e];
}

// [nrhs][n] (right-hand-side major) -> [n][B] with zero padding; node 0 (pinned) set to 0
__global__ void k_b_to_nodemajor(int n, int nrhs, int B, const double *__restrict__ in, double *__restrict__ out)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)n * B) return;
    const int i = (int)(e / B), b = (int)(e % B);
    out[e] = (b < nrhs && i != 0) ? in[(long)b * n + i] : 0.0;
}

__global__ void k_b_to_rhsmajor(int n, int nrhs, int B, const double *__restrict__ in, double *__restrict__ out)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)n * nrhs) return;
    const int b = (int)(e / n), i = (int)(e % n);
    out[e] = in[(long)i * B + b];
}

// ---------------------------------------------------------------------------
// set-up of the solve: pinned operator, diagonal, boundary list, spectral
// bounds, coarsest inverse
// ---------------------------------------------------------------------------
__global__ void k_b_pin(int n, const int *__restrict__ rp, const int *__restrict__ col, const double *__restrict__ lapP,
                        double *__restrict__ A64, float *__restrict__ A32, double *__restrict__ dinv64,
                        float *__restrict__ dinv32, int *__restrict__ nodiag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double diag = 0;
    bool found = false;
    for (int j = rp[i]; j < rp[i + 1]; j++) {
        double v = lapP[j];
        if (i == 0) v = (col[j] == 0 && !found) ? 1.0 : 0.0;
        A64[j] = v;
        A32[j] = (float)v;
        if (col[j] == i && !found) { diag = v; found = true; }
    }
    if (!found || diag == 0) atomicOr(nodiag, 1);
    dinv64[i] = diag != 0 ? 1.0 / diag : 0.0;
    dinv32[i] = (float)dinv64[i];
}

__global__ void k_b_pow(int n, const int *__restrict__ rp, const int *__restrict__ col, const double *__restrict__ A,
                        const double *__restrict__ dinv, const uint8_t *__restrict__ btag,
                        const double *__restrict__ v, double *__restrict__ w, double *__restrict__ part)
{
    __shared__ double sm[256];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double val = 0;
    if (i < n && !btag[i]) {
        double s = 0;
        for (int j = rp[i]; j < rp[i + 1]; j++) s += A[j] * v[col[j]];
        val = dinv[i] * s;
    }
    if (i < n) w[i] = val;
    sm[threadIdx.x] = val * val;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}

__global__ void k_b_seed(int n, const uint8_t *btag, double *v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    unsigned h = (unsigned)i * 2654435761u;
    h ^= h >> 16; h *= 2246822519u; h ^= h >> 13;
    v[i] = btag[i] ? 0.0 : ((double)(h & 0xffffff) / 16777216.0 - 0.5);
}

__global__ void k_b_mul(int n, double *v, double f)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] *= f;
}

// padded ELL [kmax][n] of a CSR matrix (padding: self index, zero weight)
__global__ void k_b_csr_to_ell(int n, int kmax, const int *__restrict__ rp, const int *__restrict__ col,
                               const double *__restrict__ A, int *__restrict__ idx, double *__restrict__ Ae)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int beg = rp[i], len = rp[i + 1] - beg;
    for (int j = 0; j < kmax; j++) {
        idx[(long)j * n + i] = j < len ? col[beg + j] : i;
        Ae[(long)j * n + i] = j < len ? A[beg + j] : 0.0;
    }
}

void batch_prepare_solver(mgm_batch *b)
{
    cudaStream_t s = b->s;
    DBuf<int> flag(1);
    flag.zero(s);
    for (int l = 0; l < b->nl; l++) {
        BLevel &L = b->L[l];
        const size_t nz = (size_t)std::max<long long>(L.nnz, 1);
        L.A64.alloc(nz); L.A32.alloc(nz); L.dinv64.alloc(L.n); L.dinv32.alloc(L.n);
        k_b_pin<<<blocks_for(L.n, 256), 256, 0, s>>>(L.n, L.rp.p, L.col.p, L.lapP.p, L.A64.p, L.A32.p, L.dinv64.p,
                                                     L.dinv32.p, flag.p);
        MGM_LAUNCHED();
        if (L.r_nnz > 0) { L.r_w32.alloc((size_t)L.r_nnz); convert_d2f(L.r_w64.p, L.r_w32.p, L.r_nnz, s); }
        if (L.p_nnz > 0) { L.p_w32.alloc((size_t)L.p_nnz); convert_d2f(L.p_w64.p, L.p_w32.p, L.p_nnz, s); }
        std::vector<uint8_t> hb(L.n);
        L.btag.download(hb.data(), L.n, s);
        MGM_CUDA(cudaStreamSynchronize(s));
        std::vector<int> bl;
        for (int i = 0; i < L.n; i++) if (hb[i]) bl.push_back(i);
        L.nbl = (int)bl.size();
        L.bnd_list.upload(bl.data(), bl.size(), s);
        if (l < b->nl - 1) {
            // largest eigenvalue of D^-1 A on interior rows (power iteration)
            const int nb = blocks_for(L.n, 256);
            DBuf<double> v(L.n), w(L.n), part(nb);
            std::vector<double> hp(nb);
            k_b_seed<<<nb, 256, 0, s>>>(L.n, L.btag.p, v.p);
            MGM_LAUNCHED();
            double lam = 0;
            for (int it = 0; it < 40; it++) {
                k_b_pow<<<nb, 256, 0, s>>>(L.n, L.rp.p, L.col.p, L.A64.p, L.dinv64.p, L.btag.p, v.p, w.p, part.p);
                MGM_LAUNCHED();
                part.download(hp.data(), nb, s);
                MGM_CUDA(cudaStreamSynchronize(s));
                double sq = 0;
                for (double x : hp) sq += x;
                if (it > 0) lam = sqrt(sq);
                k_b_mul<<<nb, 256, 0, s>>>(L.n, w.p, sq > 0 ? 1.0 / sqrt(sq) : 0.0);
                MGM_LAUNCHED();
                std::swap(v.p, w.p);
            }
            L.lmax = lam > 0 && std::isfinite(lam) ? lam : 2.0;
        }
    }
    int hf = 0;
    flag.download(&hf, 1, s);
    MGM_CUDA(cudaStreamSynchronize(s));
    MGM_REQUIRE(hf == 0, "mgm_batch_setup: a row of the Poisson operator has no (nonzero) diagonal entry");
    BLevel &C = b->L[b->nl - 1];
    MGM_REQUIRE(C.n <= 8192, "mgm_batch_setup: coarsest level too large for the dense solve (use more levels)");
    DBuf<int> idx((size_t)C.n * C.kmax);
    DBuf<double> Ae((size_t)C.n * C.kmax);
    k_b_csr_to_ell<<<blocks_for(C.n, 128), 128, 0, s>>>(C.n, C.kmax, C.rp.p, C.col.p, C.A64.p, idx.p, Ae.p);
    MGM_LAUNCHED();
    b->cinv64.alloc((size_t)C.n * C.n);
    b->cinv32.alloc((size_t)C.n * C.n);
    dense_inverse(C.n, C.kmax, idx.p, Ae.p, b->cinv64.p, b->cinv32.p, s);
}

void batch_free_solver(mgm_batch *b)
{
    for (int l = 0; l < kBatchMaxLevels; l++) {
        b->v64[l] = BVecs<double>();
        b->v32[l] = BVecs<float>();
    }
    b->X.release(); b->Bv.release(); b->V.release(); b->part.release(); b->hsc.release(); b->stage.release();
    b->Z32.release(); b->Z64.release();
    b->V_cols = b->Z_cols32 = b->Z_cols64 = 0;
    b->B = 0;
}

// ---------------------------------------------------------------------------
// V-cycle
// ---------------------------------------------------------------------------
namespace {

template <class T>
struct BLev {
    int n, nbl;
    const int *rp, *col, *bnd_list;
    const T *A, *dinv;
    const uint8_t *btag;
    const int *r_rp, *r_col, *p_rp, *p_col;
    const T *r_w, *p_w;
    T *r, *e, *e2, *d, *q;
    double lmax;
};

template <class T>
BVecs<T> &vecs(mgm_batch *b, int l);
template <>
BVecs<double> &vecs<double>(mgm_batch *b, int l) { return b->v64[l]; }
template <>
BVecs<float> &vecs<float>(mgm_batch *b, int l) { return b->v32[l]; }

template <class T>
std::vector<BLev<T>> blevels(mgm_batch *b)
{
    std::vector<BLev<T>> out;
    for (int l = 0; l < b->nl; l++) {
        BLevel &L = b->L[l];
        BVecs<T> &V = vecs<T>(b, l);
        BLev<T> o{};
        o.n = L.n; o.nbl = L.nbl; o.rp = L.rp.p; o.col = L.col.p; o.bnd_list = L.bnd_list.p; o.btag = L.btag.p;
        if constexpr (sizeof(T) == 8) { o.A = L.A64.p; o.dinv = L.dinv64.p; o.r_w = L.r_w64.p; o.p_w = L.p_w64.p; }
        else { o.A = L.A32.p; o.dinv = L.dinv32.p; o.r_w = L.r_w32.p; o.p_w = L.p_w32.p; }
        o.r_rp = L.r_rp.p; o.r_col = L.r_col.p; o.p_rp = L.p_rp.p; o.p_col = L.p_col.p;
        o.r = V.r.p; o.e = V.e.p; o.e2 = V.e2.p; o.d = V.d.p; o.q = V.q.p;
        o.lmax = L.lmax;
        out.push_back(o);
    }
    return out;
}


template <class T, int Q>
void bsmooth(mgm_batch *b, BLev<T> &L, bool zero_start)
{
    cudaStream_t s = b->s;
    const int B = 32 * Q;
    const double lM = 1.05 * L.lmax, lm = L.lmax / b->cheb_ratio;
    const double th = 0.5 * (lM + lm), de = 0.5 * (lM - lm), sig = th / de;
    double rho = 1.0 / sig;
    k_b_bnd<T, Q><<<rows_grid(L.nbl), 256, 0, s>>>(L.nbl, L.bnd_list, L.rp, L.col, L.A, L.dinv, L.r, L.e, B,
                                                    zero_start ? 1 : 0);
    MGM_LAUNCHED();
    for (int step = 0; step < b->cheb_deg; step++) {
        double c1 = 0, c2;
        if (step == 0) c2 = 1.0 / th;
        else {
            const double rn = 1.0 / (2.0 * sig - rho);
            c1 = rn * rho;
            c2 = 2.0 * rn / de;
            rho = rn;
        }
        k_b_cheb<T, Q><<<rows_grid(L.n), 256, 0, s>>>(L.n, L.rp, L.col, L.A, L.dinv, L.btag, L.r, L.e, L.e2, L.d,
                                                       B, (T)c1, (T)c2, step == 0 ? 1 : 0);
        MGM_LAUNCHED();
        std::swap(L.e, L.e2);
        k_b_bnd<T, Q><<<rows_grid(L.nbl), 256, 0, s>>>(L.nbl, L.bnd_list, L.rp, L.col, L.A, L.dinv, L.r, L.e, B, 0);
        MGM_LAUNCHED();
    }
}

template <class T, int Q>
void bvcycle(mgm_batch *b, std::vector<BLev<T>> &Ls, int l)
{
    cudaStream_t s = b->s;
    const int B = 32 * Q;
    BLev<T> &L = Ls[l];
    if (l == b->nl - 1) {
        const T *inv;
        if constexpr (sizeof(T) == 8) inv = b->cinv64.p; else inv = b->cinv32.p;
        k_b_dense<T, B><<<blocks_for(L.n, 32), 256, 0, s>>>(L.n, inv, L.r, L.e);
        MGM_LAUNCHED();
        return;
    }
    MGM_CUDA(cudaMemsetAsync(L.e, 0, sizeof(T) * (size_t)L.n * B, s));
    bsmooth<T, Q>(b, L, true);
    BLev<T> &C = Ls[l + 1];
    k_b_residual<T, Q><<<rows_grid(L.n), 256, 0, s>>>(L.n, L.rp, L.col, L.A, L.btag, L.r, L.e, L.q, B);
    MGM_LAUNCHED();
    k_b_restrict<T, Q><<<rows_grid(C.n), 256, 0, s>>>(C.n, C.r_rp, C.r_col, C.r_w, L.q, C.r, B);
    MGM_LAUNCHED();
    bvcycle<T, Q>(b, Ls, l + 1);
    k_b_prolong<T, Q><<<rows_grid(L.n), 256, 0, s>>>(L.n, L.p_rp, L.p_col, L.p_w, C.e, L.e, B);
    MGM_LAUNCHED();
    bsmooth<T, Q>(b, L, false);
}

template <class T>
void ensure_vecs(mgm_batch *b, int B, int m)
{
    if (b->B != B) batch_free_solver(b);
    b->B = B;
    for (int l = 0; l < b->nl; l++) {
        BVecs<T> &V = vecs<T>(b, l);
        const size_t nB = (size_t)b->L[l].n * B;
        if (V.r.n != nB) for (DBuf<T> *x : {&V.r, &V.e, &V.e2, &V.d, &V.q}) { x->alloc(nB); x->zero(b->s); }
    }
    const size_t nB = (size_t)b->L[0].n * B;
    if (b->X.n != nB) { b->X.alloc(nB); b->Bv.alloc(nB); }
    if (b->V_cols < m + 1) { b->V.alloc(nB * (m + 1)); b->V_cols = m + 1; }
    if constexpr (sizeof(T) == 4) { if (b->Z_cols32 < m) { b->Z32.alloc(nB * m); b->Z_cols32 = m; } }
    else { if (b->Z_cols64 < m) { b->Z64.alloc(nB * m); b->Z_cols64 = m; } }
    const size_t need = (size_t)(3 * (kBatchMaxRestart + 2)) * 64 + 64;
    if (b->h_pinned_n < need) {
        if (b->h_pinned) cudaFreeHost(b->h_pinned);
        b->h_pinned = nullptr;
        MGM_CUDA(cudaMallocHost(&b->h_pinned, need * sizeof(double)));
        b->h_pinned_n = need;
    }
    if (b->hsc.n < need) b->hsc.alloc(need);
}

int dot_grid(long n) { return (int)std::max(1L, std::min<long>((n + 7) / 8, 148L * 8)); }

template <class T, int Q>
void bfgmres(mgm_batch *b, int nrhs, int *vcycles, double *rel_res)
{
    cudaStream_t s = b->s;
    const int B = 32 * Q;
    BLevel &L0 = b->L[0];
    const int n = L0.n;
    const long nB = (long)n * B;
    const int m = std::min(b->restart, kBatchMaxRestart);
    auto Ls = blevels<T>(b);
    T *Z;
    if constexpr (sizeof(T) == 8) Z = b->Z64.p; else Z = b->Z32.p;
    double *V = b->V.p, *X = b->X.p, *hp = b->h_pinned, *dsc = b->hsc.p;
    const int gres = dot_grid(n);
    const int gdot = (int)std::max(1L, std::min<long>((n + (256 / B) - 1) / (256 / B), 148L * 8));
    const size_t part_need = std::max({(size_t)gres * 2 * B, (size_t)gdot * 8 * B, (size_t)148 * 16 * B});
    if (b->part.n < part_need) b->part.alloc(part_need);
    std::vector<double> bnorm(B, 0.0), relres(B, 0.0);
    std::vector<double> H((size_t)B * (m + 1) * m), cs((size_t)B * m), sn((size_t)B * m), g((size_t)B * (m + 1));
    long long vc = 0;
    const int max_restarts = b->max_restarts;
    // reduction helper: part (gridblocks x cnt x B) -> dsc[off ...] -> host hp[off ...]
    auto multidot = [&](int cnt, const double *Vb, const double *Wv, int off) {
        for (int c0 = 0; c0 < cnt; c0 += 8) {
            const int cc = std::min(8, cnt - c0);
            k_b_multidot<<<gdot, 256, 0, s>>>(n, B, cc, Vb + (long)c0 * nB, nB, Wv, b->part.p);
            MGM_LAUNCHED();
            k_b_reduce<<<cc * ((B + 31) / 32), 256, 0, s>>>(b->part.p, gdot, cc, B, dsc + off + c0 * B);
            MGM_LAUNCHED();
        }
    };
    for (int restart = 0; restart <= max_restarts; restart++) {
        k_b_resid64<double, Q><<<gres, 256, 0, s>>>(n, L0.rp.p, L0.col.p, L0.A64.p, b->Bv.p, X, V, b->part.p, B);
        MGM_LAUNCHED();
        k_b_reduce<<<2 * ((B + 31) / 32), 256, 0, s>>>(b->part.p, gres, 2, B, dsc);
        MGM_LAUNCHED();
        MGM_CUDA(cudaMemcpyAsync(hp, dsc, sizeof(double) * 2 * B, cudaMemcpyDeviceToHost, s));
        MGM_CUDA(cudaStreamSynchronize(s));
        bool active = false;
        for (int q = 0; q < B; q++) {
            bnorm[q] = sqrt(hp[B + q]);
            const double beta = sqrt(hp[q]);
            relres[q] = bnorm[q] > 0 ? beta / bnorm[q] : 0.0;
            if (!std::isfinite(relres[q])) throw Error{MGM_ERR_DIVERGED, "batched Poisson solve: non-finite residual"};
            if (q < nrhs && bnorm[q] > 0 && relres[q] >= b->tol) active = true;
            hp[q] = beta;
        }
        if (!active || restart == max_restarts) break;
        MGM_CUDA(cudaMemcpyAsync(dsc, hp, sizeof(double) * B, cudaMemcpyHostToDevice, s));
        k_b_scale<<<blocks_for(nB, 256), 256, 0, s>>>(nB, B, V, V, dsc, 0);
        MGM_LAUNCHED();
        std::fill(g.begin(), g.end(), 0.0);
        for (int q = 0; q < B; q++) g[(size_t)q * (m + 1)] = hp[q];
        int j_done = 0;
        for (int j = 0; j < m; j++) {
            BLev<T> &F = Ls[0];
            k_b_convert<double, T><<<blocks_for(nB, 256), 256, 0, s>>>(nB, V + (long)j * nB, F.r);
            MGM_LAUNCHED();
            std::vector<BLev<T>> cyc = Ls;
            bvcycle<T, Q>(b, cyc, 0);
            vc++;
            k_b_convert<T, T><<<blocks_for(nB, 256), 256, 0, s>>>(nB, cyc[0].e, Z + (long)j * nB);
            MGM_LAUNCHED();
            // w = A z_j, written into the slot of V_{j+1}; classical Gram-Schmidt with
            // the norm of w in the same pass, a second pass only when the first one
            // cancelled more than 1 - 1/sqrt(2) of |w| for some right-hand side
            // (the Daniel-Gragg-Kaufman-Stewart test)
            double *Wn = V + (long)(j + 1) * nB;
            k_b_apply64<T, Q><<<rows_grid(n), 256, 0, s>>>(n, L0.rp.p, L0.col.p, L0.A64.p, Z + (long)j * nB, Wn, B);
            MGM_LAUNCHED();
            const int h1 = 0, h2 = (kBatchMaxRestart + 2) * B, h3 = 2 * (kBatchMaxRestart + 2) * B;
            multidot(j + 2, V, Wn, h1);  // dots with V_0..V_j, then |w|^2
            const int gorth = (int)std::min<long>(blocks_for(nB, 256), 148L * 16);
            k_b_orth_norm<<<gorth, 256, 0, s>>>(nB, B, j + 1, V, nB, dsc + h1, Wn, b->part.p);
            MGM_LAUNCHED();
            k_b_reduce<<<(B + 31) / 32, 256, 0, s>>>(b->part.p, gorth, 1, B, dsc + h3);
            MGM_LAUNCHED();
            MGM_CUDA(cudaMemcpyAsync(hp, dsc, sizeof(double) * (h3 + B), cudaMemcpyDeviceToHost, s));
            MGM_CUDA(cudaStreamSynchronize(s));
            bool again = false;
            for (int q = 0; q < B; q++)
                if (hp[h3 + q] < 0.5 * hp[h1 + (j + 1) * B + q]) again = true;
            for (int i = 0; i <= j; i++) for (int q = 0; q < B; q++) hp[h2 + i * B + q] = 0.0;
            if (again) {
                multidot(j + 1, V, Wn, h2);
                k_b_orth_norm<<<gorth, 256, 0, s>>>(nB, B, j + 1, V, nB, dsc + h2, Wn, b->part.p);
                MGM_LAUNCHED();
                k_b_reduce<<<(B + 31) / 32, 256, 0, s>>>(b->part.p, gorth, 1, B, dsc + h3);
                MGM_LAUNCHED();
                MGM_CUDA(cudaMemcpyAsync(hp + h2, dsc + h2, sizeof(double) * (h3 - h2 + B), cudaMemcpyDeviceToHost, s));
                MGM_CUDA(cudaStreamSynchronize(s));
            }
            k_b_scale<<<blocks_for(nB, 256), 256, 0, s>>>(nB, B, Wn, Wn, dsc + h3, 1);
            MGM_LAUNCHED();
            double worst = 0;
            for (int q = 0; q < B; q++) {
                double *col = &H[((size_t)q * m + j) * (m + 1)];
                double *csq = &cs[(size_t)q * m], *snq = &sn[(size_t)q * m], *gq = &g[(size_t)q * (m + 1)];
                for (int i = 0; i <= j; i++) col[i] = hp[h1 + i * B + q] + hp[h2 + i * B + q];
                col[j + 1] = sqrt(std::max(hp[h3 + q], 0.0));
                for (int i = 0; i < j; i++) {
                    const double t0 = csq[i] * col[i] + snq[i] * col[i + 1];
                    col[i + 1] = -snq[i] * col[i] + csq[i] * col[i + 1];
                    col[i] = t0;
                }
                const double a = col[j], c = col[j + 1];
                const double rden = std::hypot(a, c);
                csq[j] = rden > 0 ? a / rden : 1.0;
                snq[j] = rden > 0 ? c / rden : 0.0;
                col[j] = rden;
                col[j + 1] = 0;
                gq[j + 1] = -snq[j] * gq[j];
                gq[j] = csq[j] * gq[j];
                if (q < nrhs && bnorm[q] > 0) {
                    const double est = fabs(gq[j + 1]) / bnorm[q];
                    if (!std::isfinite(est)) throw Error{MGM_ERR_DIVERGED, "batched Poisson solve: non-finite Krylov residual"};
                    worst = std::max(worst, est);
                }
            }
            j_done = j + 1;
            if (worst < b->tol) break;
        }
        // per right-hand side: y = H^-1 g, X += Z y
        for (int q = 0; q < B; q++) {
            const double *Hq = &H[(size_t)q * m * (m + 1)];
            const double *gq = &g[(size_t)q * (m + 1)];
            std::vector<double> y(j_done, 0.0);
            for (int i = j_done - 1; i >= 0; i--) {
                double acc = gq[i];
                for (int c = i + 1; c < j_done; c++) acc -= Hq[(size_t)c * (m + 1) + i] * y[c];
                const double dgn = Hq[(size_t)i * (m + 1) + i];
                y[i] = dgn != 0 ? acc / dgn : 0.0;
            }
            for (int i = 0; i < j_done; i++) hp[i * B + q] = y[i];
        }
        MGM_CUDA(cudaMemcpyAsync(dsc, hp, sizeof(double) * j_done * B, cudaMemcpyHostToDevice, s));
        k_b_combine<T><<<blocks_for(nB, 256), 256, 0, s>>>(nB, B, j_done, Z, nB, dsc, X);
        MGM_LAUNCHED();
    }
    double worst = 0;
    for (int q = 0; q < nrhs; q++) { rel_res[q] = relres[q]; worst = std::max(worst, relres[q]); }
    *vcycles = (int)vc;
    if (!(worst < b->tol))
        throw Error{MGM_ERR_DIVERGED, "batched Poisson solve did not reach the tolerance (worst rel. residual " +
                                          std::to_string(worst) + " after " + std::to_string(vc) + " V-cycles)"};
}

}  // namespace

void batch_solve(mgm_batch *b, int mode, int nrhs, const double *rhs_host, double *sol_host, int *vcycles,
                 double *rel_res, double *solve_ms)
{
    MGM_REQUIRE(b->setup_done, "mgm_batch_solve: call mgm_batch_setup first");
    MGM_REQUIRE(nrhs >= 1 && nrhs <= 64, "mgm_batch_solve: nrhs must be in [1, 64]");
    MGM_REQUIRE(mode == MGM_MODE_FP64 || mode == MGM_MODE_FP32_IR, "mgm_batch_solve: mode must be MGM_MODE_FP64 or MGM_MODE_FP32_IR");
    cudaStream_t s = b->s;
    const int B = nrhs <= 32 ? 32 : 64;
    const int m = std::min(b->restart, kBatchMaxRestart);
    if (mode == MGM_MODE_FP64) ensure_vecs<double>(b, B, m); else ensure_vecs<float>(b, B, m);
    const int n = b->L[0].n;
    // staging buffer kept across solves (no allocation per solve); the copies
    // run at page-locked speed when the caller's buffers are page-locked
    if (b->stage.n < (size_t)n * nrhs) b->stage.alloc((size_t)n * nrhs);
    DBuf<double> &hbuf = b->stage;
    MGM_CUDA(cudaMemcpyAsync(hbuf.p, rhs_host, sizeof(double) * (size_t)n * nrhs, cudaMemcpyHostToDevice, s));
    for (int q = 0; q < 4; q++) if (!b->ev[q]) MGM_CUDA(cudaEventCreate(&b->ev[q]));
    k_b_to_nodemajor<<<blocks_for((long)n * B, 256), 256, 0, s>>>(n, nrhs, B, hbuf.p, b->Bv.p);
    MGM_LAUNCHED();
    MGM_CUDA(cudaMemsetAsync(b->X.p, 0, sizeof(double) * (size_t)n * B, s));
    MGM_CUDA(cudaEventRecord(b->ev[0], s));
    if (mode == MGM_MODE_FP64) {
        if (B == 32) bfgmres<double, 1>(b, nrhs, vcycles, rel_res); else bfgmres<double, 2>(b, nrhs, vcycles, rel_res);
    } else {
        if (B == 32) bfgmres<float, 1>(b, nrhs, vcycles, rel_res); else bfgmres<float, 2>(b, nrhs, vcycles, rel_res);
    }
    MGM_CUDA(cudaEventRecord(b->ev[1], s));
    k_b_to_rhsmajor<<<blocks_for((long)n * nrhs, 256), 256, 0, s>>>(n, nrhs, B, b->X.p, hbuf.p);
    MGM_LAUNCHED();
    MGM_CUDA(cudaMemcpyAsync(sol_host, hbuf.p, sizeof(double) * (size_t)n * nrhs, cudaMemcpyDeviceToHost, s));
    MGM_CUDA(cudaStreamSynchronize(s));
    float ms = 0;
    MGM_CUDA(cudaEventElapsedTime(&ms, b->ev[0], b->ev[1]));
    if (solve_ms) *solve_ms = ms;
}

}  // namespace mgm
