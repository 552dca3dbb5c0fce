// solver.cu -- convergent Poisson solve for the pinned system
//     A p = b,  A = lap_Poison with row 0 replaced by p[0] = 0,
// the system whose solution the reference's multigrid_Poisson_solver
// (fractional_step_solver.h:150-196, p -= p[0] after each sweep) aims at.
//
// Preconditioner: one V-cycle in precision T (double or float)
//   smoother   Chebyshev polynomial in D^-1 A on interior rows, every step
//              followed by an exact solve of the boundary rows (a boundary
//              row couples only to itself and interior nodes, kdtree_functions.h:141-149);
//   transfer   interior residuals restricted with the RBF interpolation
//              weights of create_restriction_matrix (mesh_functions.h:533-600)
//              built for every non-boundary coarse row; corrections prolongated
//              with create_prolongation_matrix weights (mesh_functions.h:602-670)
//              built for every fine row, shifted so the pinned node gets none;
//   coarsest   dense inverse of the pinned coarsest operator.
// Outer: flexible GMRES in FP64 (residuals, Krylov basis, solution updates).
#include <cmath>

#include "stencil.cuh"

namespace mgm {

template <int BS>
__device__ __forceinline__ double block_sum_d(double v, double *sm)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < BS / 32 ? sm[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();
    return v;
}

// ---------------------------------------------------------------------------
// smoother
// ---------------------------------------------------------------------------
// Row work of the V-cycle kernels, shared by the one-operation kernels and
// the fused coarse-level V-cycle (k_coarse_vcycle), which therefore give the
// same bits.  COH: the vectors (r, e, d, q) are loaded from L2, past the
// SM's L1 and the read-only path -- in the fused kernel other CTAs rewrite
// them between passes; the operators are read-only throughout.
template <bool COH, class T>
__device__ __forceinline__ T ldv(const T *p)
{
    if constexpr (COH) return __ldcg(p);
    else return *p;
}

template <class T, bool COH = false>
__device__ __forceinline__ void start_row(int i, const uint8_t *__restrict__ btag, const T *__restrict__ dinv,
                                          const T *r, T *e)
{
    e[i] = btag[i] ? ldv<COH>(r + i) * dinv[i] : T(0);
}
// boundary row w of the list, by the 32 lanes of a warp
template <class T, bool COH = false>
__device__ __forceinline__ void bnd_row_warp(int w, int lane, const int *__restrict__ list, int k,
                                             const int *__restrict__ bidx, const T *__restrict__ bA,
                                             const T *__restrict__ dinv, const T *r, T *e)
{
    const int i = list[w];
    T s = T(0);
    for (int j = lane; j < k; j += 32) s += bA[(long)w * k + j] * ldv<COH>(e + bidx[(long)w * k + j]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) e[i] = ldv<COH>(e + i) + (ldv<COH>(r + i) - s) * dinv[i];
}

// Start of a smoothing pass from e = 0: interior rows 0, boundary rows their
// exact solve r_i / a_ii (they couple only to interior nodes).
template <class T>
__global__ void __launch_bounds__(256) k_start_e(int n, const uint8_t *__restrict__ btag, const T *__restrict__ dinv,
                                                 const T *__restrict__ r, T *__restrict__ e)
{
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) start_row(i, btag, dinv, r, e);
}

// Exact solve of the boundary rows, one warp per row.  A boundary row couples
// only to itself and interior nodes, so rows can be updated in place.  The
// rows are stored compactly (row-major [nbl][k]) so that a warp reads them
// with coalesced loads.
template <class T>
__global__ void __launch_bounds__(256) k_bnd_exact(int nbl, const int *__restrict__ list, int k,
                                                   const int *__restrict__ bidx, const T *__restrict__ bA,
                                                   const T *__restrict__ dinv, const T *__restrict__ r,
                                                   T *__restrict__ e)
{
    pdl_enter();
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= nbl) return;
    bnd_row_warp(w, lane, list, k, bidx, bA, dinv, r, e);
}

// One Chebyshev step on interior rows: q = r - A e, d = c1*d + c2*D^-1 q, e' = e + d.
// Boundary rows copy e.  zero_start: e is zero except on boundary rows.
template <class T>
__global__ void __launch_bounds__(256) k_cheb(int n, int ld, int k, const int *__restrict__ idx, const T *__restrict__ A,
                                              const T *__restrict__ dinv, const uint8_t *__restrict__ btag,
                                              const T *__restrict__ r, const T *__restrict__ e, T *__restrict__ eout,
                                              T *__restrict__ d, T c1, T c2, int first)
{
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const T ei = e[i];
    if (btag[i]) { eout[i] = ei; return; }
    const T q = r[i] - ell_row_dot(idx, A, e, ld, k, i);
    const T di = first ? c2 * dinv[i] * q : c1 * d[i] + c2 * dinv[i] * q;
    d[i] = di;
    eout[i] = ei + di;
}

// residual on interior rows (boundary rows are solved exactly: 0)
template <class T>
__global__ void __launch_bounds__(256) k_residual(int n, int ld, int k, const int *__restrict__ idx,
                                                  const T *__restrict__ A, const uint8_t *__restrict__ btag,
                                                  const T *__restrict__ r, const T *__restrict__ e, T *__restrict__ q)
{
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (btag[i]) { q[i] = T(0); return; }
    q[i] = r[i] - ell_row_dot(idx, A, e, ld, k, i);
}

// coarse rhs: r_c[i] = sum_j Rw[j][i] q_f[Ridx[j][i]] on interior coarse rows, 0 elsewhere
template <class T>
__global__ void __launch_bounds__(256) k_restrict(int n, int k, const int *__restrict__ ridx, const T *__restrict__ rw,
                                                  const uint8_t *__restrict__ btag, const T *__restrict__ qf,
                                                  T *__restrict__ rc)
{
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (btag[i] || i == 0) { rc[i] = T(0); return; }
    rc[i] = ell_row_dot(ridx, rw, qf, n, k, i);
}

// (P e_c)[0], the prolongated correction at the pinned node, by the 32 lanes
// of warp 0: the lanes fetch the operands of 32 slots at once (operand(j, a,
// x): weight and gathered value of slot j), then every lane sums the
// products in slot order, one fused multiply-add per slot -- the rounding of
// the row dots (ell_row_dot, ell_row_dot_o), so the shift has the bits a
// serial row-0 dot would give.
template <class T, class Op>
__device__ __forceinline__ T row0_dot_warp(int k, Op operand)
{
    const int lane = threadIdx.x & 31;
    T s = T(0);
    for (int j0 = 0; j0 < k; j0 += 32) {
        T a = T(0), x = T(0);
        if (j0 + lane < k) operand(j0 + lane, a, x);
        const int m = min(32, k - j0);
        for (int q = 0; q < m; q++) s = fma_rn(__shfl_sync(0xffffffffu, a, q), __shfl_sync(0xffffffffu, x, q), s);
    }
    return s;
}

// e_f[i] += (P e_c)[i] - (P e_c)[0]  (the shift keeps the pinned node uncorrected)
template <class T>
__global__ void __launch_bounds__(256) k_prolong(int n, int k, const int *__restrict__ pidx, const T *__restrict__ pw,
                                                 const T *__restrict__ ec, T *__restrict__ ef)
{
    pdl_enter();
    __shared__ T shift;
    if (threadIdx.x < 32) {
        const T s = row0_dot_warp<T>(k, [&](int j, T &a, T &x) {
            a = pw[(long)j * n];
            x = ec[pidx[(long)j * n]];
        });
        if (threadIdx.x == 0) shift = s;
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ef[i] += ell_row_dot(pidx, pw, ec, n, k, i) - shift;
}

// ---------------------------------------------------------------------------
// compact FP32 path: FP32 weights, neighbours stored as int16 offsets c - base
// (6 bytes per stencil slot instead of 8)
// ---------------------------------------------------------------------------
// The gathered vector x is read through the read-only path unless COHERENT
// (the fused coarse V-cycle, where other CTAs rewrite x between passes).
template <class T, class X, bool COHERENT = false>
__device__ __forceinline__ T ell_row_dot_o(const short *__restrict__ off, const T *__restrict__ A,
                                           const X *__restrict__ x, long n, int k, long i, int base)
{
    T s = T(0);
    int j = 0;
    for (; j + 8 <= k; j += 8) {
        int c[8];
        T a[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const long o = (long)(j + q) * n + i;
            c[q] = base + (int)__ldg(off + o);
            a[q] = __ldg(A + o);
        }
#pragma unroll
        for (int q = 0; q < 8; q++) s = fma_rn(a[q], (T)(COHERENT ? __ldcg(x + c[q]) : __ldg(x + c[q])), s);
    }
    for (; j < k; j++) {
        const long o = (long)j * n + i;
        s = fma_rn(A[o], (T)ldv<COHERENT>(x + base + (int)off[o]), s);
    }
    return s;
}

// Compact level kernels (FP32 or FP64 weights, int16 offsets, ELL [k][ld],
// each row's slots sorted by neighbour index).
//
// k_level_v4: four consecutive rows per thread; the weights and offsets of
// rows i0..i0+3 come in as one 16-byte (FP32; two for FP64) and one 8-byte
// load per stencil slot (ld a multiple of 4; streamed past L1 with
// evict-first loads), so a thread has 8 operator loads and 16 gathers in
// flight per 4 slots.  For the large levels, which are bandwidth-bound.
// k_level_c1: one row per thread, for the small levels, which are latency-
// bound and need the threads more than the wide loads.
// Each row's sum runs in slot order in both, as in every other level kernel
// of the same precision, so all of them give the same bits.  MODE 0:
// Chebyshev step q = r - A e, d = c1 d + c2 D^-1 q, e' = e + d on interior
// rows (boundary rows copy e); MODE 1: residual q = r - A e on interior rows,
// 0 on boundary rows.
template <int MODE, class T, bool COH = false>
__device__ __forceinline__ void level_row_out(int i, T s, const T *__restrict__ dinv,
                                              const uint8_t *__restrict__ btag, const T *r, const T *e, T *out, T *d,
                                              T c1, T c2, int first)
{
    if (MODE == 0) {
        const T ei = ldv<COH>(e + i);
        if (btag[i]) { out[i] = ei; return; }
        const T q = ldv<COH>(r + i) - s;
        const T di = first ? c2 * dinv[i] * q : c1 * ldv<COH>(d + i) + c2 * dinv[i] * q;
        d[i] = di;
        out[i] = ei + di;
    } else {
        out[i] = btag[i] ? T(0) : ldv<COH>(r + i) - s;
    }
}

template <int MODE, class T, bool COHERENT = false>
__device__ __forceinline__ void c1_row(int i, int ld, int k, const short *__restrict__ off, const T *__restrict__ A,
                                       const T *__restrict__ dinv, const uint8_t *__restrict__ btag,
                                       const T *__restrict__ r, const T *__restrict__ e, T *__restrict__ out,
                                       T *__restrict__ d, T c1, T c2, int first)
{
    if (btag[i]) {
        out[i] = MODE == 0 ? ldv<COHERENT>(e + i) : T(0);
        return;
    }
    level_row_out<MODE, T, COHERENT>(i, ell_row_dot_o<T, T, COHERENT>(off, A, e, ld, k, i, i), dinv, btag, r, e, out,
                                     d, c1, c2, first);
}

template <int MODE, class T>
__global__ void __launch_bounds__(256) k_level_c1(int n, int ld, int k, const short *__restrict__ off,
                                                  const T *__restrict__ A, const T *__restrict__ dinv,
                                                  const uint8_t *__restrict__ btag, const T *__restrict__ r,
                                                  const T *__restrict__ e, T *__restrict__ out,
                                                  T *__restrict__ d, T c1, T c2, int first)
{
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    c1_row<MODE, T>(i, ld, k, off, A, dinv, btag, r, e, out, d, c1, c2, first);
}

// the four weights of rows i0..i0+3 in slot o (evict-first)
__device__ __forceinline__ void load4(const float *A, long o, float (&a)[4])
{
    const float4 v = __ldcs(reinterpret_cast<const float4 *>(A + o));
    a[0] = v.x; a[1] = v.y; a[2] = v.z; a[3] = v.w;
}
__device__ __forceinline__ void load4(const double *A, long o, double (&a)[4])
{
    const double2 v0 = __ldcs(reinterpret_cast<const double2 *>(A + o));
    const double2 v1 = __ldcs(reinterpret_cast<const double2 *>(A + o + 2));
    a[0] = v0.x; a[1] = v0.y; a[2] = v1.x; a[3] = v1.y;
}

// FP32: 4 CTAs of 256 per SM (64 registers); FP64: 3 (twice the weight registers)
template <int MODE, class T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 3) k_level_v4(
    int n, int ld, int k, const short *__restrict__ off, const T *__restrict__ A, const T *__restrict__ dinv,
    const uint8_t *__restrict__ btag, const T *__restrict__ r, const T *__restrict__ e, T *__restrict__ out,
    T *__restrict__ d, T c1, T c2, int first)
{
    pdl_enter();
    const int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    if (i0 >= n) return;
    T s[4] = {T(0), T(0), T(0), T(0)};
    int j = 0;
    for (; j + 4 <= k; j += 4) {
        T a[4][4];
        int c[4][4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const long o = (long)(j + q) * ld + i0;
            load4(A, o, a[q]);
            const uint2 ov = __ldcs(reinterpret_cast<const uint2 *>(off + o));
            c[q][0] = i0 + (int)(short)(ov.x & 0xffffu);
            c[q][1] = i0 + 1 + (int)(short)(ov.x >> 16);
            c[q][2] = i0 + 2 + (int)(short)(ov.y & 0xffffu);
            c[q][3] = i0 + 3 + (int)(short)(ov.y >> 16);
        }
        // padding rows (i >= n) carry weight 0 and offset 0: clamp their gathers into the vector
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
            for (int v = 0; v < 4; v++) s[v] += a[q][v] * __ldg(e + min(c[q][v], n - 1));
    }
    for (; j < k; j++) {
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const long o = (long)j * ld + i0 + v;
            s[v] += __ldcs(A + o) * __ldg(e + min(i0 + v + (int)__ldcs(off + o), n - 1));
        }
    }
#pragma unroll
    for (int v = 0; v < 4; v++)
        if (i0 + v < n) level_row_out<MODE, T>(i0 + v, s[v], dinv, btag, r, e, out, d, c1, c2, first);
}

// k_level_h4: k_level_v4 on the FP16 operator W ~ D^-1 A, four rows per
// thread interleaved: lane t of warp g holds rows 128 g + t + 32 v (v =
// 0..3), so that a warp's gathers for one slot and row set v come from 32
// consecutive rows and its per-row loads and stores are coalesced (measured
// 8% faster than consecutive rows here; k_level_v4 measured 4% slower with
// it).  One 16-byte load per stencil slot brings the four rows' weights
// (FP16) and offsets (int16):
// 4 bytes per slot instead of 6.  The off-diagonal weights enter in
// difference form, s = sum_{j != i} w_ij (e_j - e_i) + rho_i e_i, where the
// diagonal slot (offset 0) holds rho_i, the row sum of D^-1 A: the rows then
// keep their sums (a Laplacian row maps constants to ~0) whatever the FP16
// rounding of the single weights, which would otherwise perturb the smooth
// modes by (rounding error) x (condition number).  Sums in FP32, in slot
// order.  MODE 0: d = c1 d + c2 (D^-1 r - s), e' = e + d on interior rows;
// MODE 1: q = r - s / D^-1 on interior rows, 0 on boundary rows.
template <int MODE>
__device__ __forceinline__ void level_row_out_h(int i, float s, const float *__restrict__ dinv,
                                                const uint8_t *__restrict__ btag, const float *__restrict__ r,
                                                float ei, float *__restrict__ out, float *__restrict__ d, float c1,
                                                float c2, int first)
{
    if (MODE == 0) {
        if (btag[i]) { out[i] = ei; return; }
        const float q = dinv[i] * r[i] - s;
        const float di = first ? c2 * q : c1 * d[i] + c2 * q;
        d[i] = di;
        out[i] = ei + di;
    } else {
        out[i] = btag[i] ? 0.f : r[i] - s / dinv[i];
    }
}

__device__ __forceinline__ float h16(unsigned bits) { return __half2float(__ushort_as_half((unsigned short)bits)); }

template <int MODE>
__global__ void __launch_bounds__(256, 4) k_level_h4(int n, int ld, int k, const uint4 *__restrict__ W,
                                                  const float *__restrict__ dinv, const uint8_t *__restrict__ btag,
                                                  const float *__restrict__ r, const float *__restrict__ e,
                                                  float *__restrict__ out, float *__restrict__ d, float c1, float c2,
                                                  int first)
{
    pdl_enter();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int ib = (t >> 5) * 128 + (t & 31);   // rows ib + 32 v, v = 0..3
    if (ib >= n) return;
    const long q4 = ld >> 2;
    float s[4] = {0.f, 0.f, 0.f, 0.f}, ws[4] = {0.f, 0.f, 0.f, 0.f};
    int j = 0;
    for (; j + 4 <= k; j += 4) {
        uint4 w[4];
#pragma unroll
        for (int q = 0; q < 4; q++) w[q] = __ldcs(W + (long)(j + q) * q4 + t);
        float a[4][4];
        int o[4][4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            a[q][0] = h16(w[q].x & 0xffffu); a[q][1] = h16(w[q].x >> 16);
            a[q][2] = h16(w[q].y & 0xffffu); a[q][3] = h16(w[q].y >> 16);
            o[q][0] = (int)(short)(w[q].z & 0xffffu); o[q][1] = (int)(short)(w[q].z >> 16);
            o[q][2] = (int)(short)(w[q].w & 0xffffu); o[q][3] = (int)(short)(w[q].w >> 16);
        }
        // padding rows (i >= n) carry weight 0 and offset 0: clamp their gathers into the vector
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
            for (int v = 0; v < 4; v++) {
                s[v] += a[q][v] * __ldg(e + min(ib + 32 * v + o[q][v], n - 1));
                ws[v] += o[q][v] != 0 ? a[q][v] : 0.f;
            }
    }
    for (; j < k; j++) {
        const uint4 w = __ldcs(W + (long)j * q4 + t);
#pragma unroll
        for (int v = 0; v < 4; v++) {
            const unsigned hw = (v < 2 ? w.x : w.y) >> (16 * (v & 1)), ow = (v < 2 ? w.z : w.w) >> (16 * (v & 1));
            const float a = h16(hw & 0xffffu);
            const int o = (int)(short)(ow & 0xffffu);
            s[v] += a * __ldg(e + min(ib + 32 * v + o, n - 1));
            ws[v] += o != 0 ? a : 0.f;
        }
    }
#pragma unroll
    for (int v = 0; v < 4; v++) {
        const int i = ib + 32 * v;
        if (i < n) {
            const float ei = e[i];
            level_row_out_h<MODE>(i, s[v] - ws[v] * ei, dinv, btag, r, ei, out, d, c1, c2, first);
        }
    }
}

template <int MODE, class T>
static void launch_compact(const SolveLevel<T> &L, const T *e, T *out, T c1, T c2, int first, cudaStream_t s,
                           Chain &launch)
{
    if constexpr (sizeof(T) == 4) {
        if (L.W16) {
            launch(k_level_h4<MODE>, blocks_for(L.ldi / 4, 256), 256, 0, s, L.n, L.ldi, L.k, L.W16, L.dinv, L.btag,
                     L.r, e, out, L.d, c1, c2, first);
            return;
        }
    }
    if (L.n >= kVecMinRows)
        launch(k_level_v4<MODE, T>, blocks_for((L.n + 3) / 4, 256), 256, 0, s, L.n, L.ld, L.k, L.off, L.A, L.dinv,
               L.btag, L.r, e, out, L.d, c1, c2, first);
    else
        launch(k_level_c1<MODE, T>, blocks_for(L.n, 256), 256, 0, s, L.n, L.ld, L.k, L.off, L.A, L.dinv, L.btag,
               L.r, e, out, L.d, c1, c2, first);
}

template <class T, bool COHERENT = false>
__device__ __forceinline__ void restrict_row(int i, int n, int k, const short *__restrict__ off,
                                             const int *__restrict__ base, const T *__restrict__ rw,
                                             const uint8_t *__restrict__ btag, const T *__restrict__ qf,
                                             T *__restrict__ rc)
{
    if (btag[i] || i == 0) { rc[i] = T(0); return; }
    rc[i] = ell_row_dot_o<T, T, COHERENT>(off, rw, qf, n, k, i, base[i]);
}
// (P e_c)[0] of the compact prolongation, by warp 0 of a CTA (row0_dot_warp)
template <class T, bool COH = false>
__device__ __forceinline__ T prolong_shift_warp(int n, int k, const short *__restrict__ off,
                                                const int *__restrict__ base, const T *__restrict__ pw, const T *ec)
{
    const int b0 = base[0];
    return row0_dot_warp<T>(k, [&](int j, T &a, T &x) {
        a = pw[(long)j * n];
        x = ldv<COH>(ec + b0 + (int)off[(long)j * n]);
    });
}
template <class T, bool COHERENT = false>
__device__ __forceinline__ void prolong_row(int i, int n, int k, const short *__restrict__ off,
                                            const int *__restrict__ base, const T *__restrict__ pw, const T *ec, T *ef,
                                            T shift)
{
    ef[i] = ldv<COHERENT>(ef + i) + (ell_row_dot_o<T, T, COHERENT>(off, pw, ec, n, k, i, base[i]) - shift);
}

template <class T>
__global__ void __launch_bounds__(256) k_restrict_o(int n, int k, const short *__restrict__ off,
                                                    const int *__restrict__ base, const T *__restrict__ rw,
                                                    const uint8_t *__restrict__ btag, const T *__restrict__ qf,
                                                    T *__restrict__ rc)
{
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    restrict_row(i, n, k, off, base, rw, btag, qf, rc);
}

template <class T>
__global__ void __launch_bounds__(256) k_prolong_o(int n, int k, const short *__restrict__ off,
                                                   const int *__restrict__ base, const T *__restrict__ pw,
                                                   const T *__restrict__ ec, T *__restrict__ ef)
{
    pdl_enter();
    __shared__ T shift;
    if (threadIdx.x < 32) {
        const T s = prolong_shift_warp(n, k, off, base, pw, ec);
        if (threadIdx.x == 0) shift = s;
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    prolong_row(i, n, k, off, base, pw, ec, ef, shift);
}

// ---------------------------------------------------------------------------
// tile-streamed level kernels (FP32 compact operator)
//
// The operator is stored tile-major ([tile][k][kTileRows]: a tile's weights,
// and separately its int16 offsets, are contiguous).  A persistent CTA walks
// tiles of kTileRows rows; for each tile one thread issues two bulk
// asynchronous copies (cp.async.bulk, the TMA engine's 1-D form) into shared
// memory, completing on an mbarrier; two stages alternate, so the next tile's
// operator streams in while this tile's rows gather their neighbours.  A
// thread then reads its row's stencil from shared memory and issues its
// neighbour gathers back to back.  The products are summed in slot order, as
// in k_level_v4, so the results are the same bits.
//
// Every mbarrier wait is bounded: on time-out the CTA sets *err, waits (again
// bounded) for the copies it still has in flight, and stops.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity)
{
    for (int it = 0; it < (1 << 20); it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// global -> shared bulk copy; addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// One pipeline stage in shared memory: the tile's weights [k][kTileRows] f32
// and offsets [k][kTileRows] i16.
struct TileStage {
    int k;
    __device__ size_t a_off() const { return 0; }
    __device__ size_t o_off() const { return (size_t)k * kTileRows * sizeof(float); }
    __device__ size_t bytes() const { return (size_t)k * kTileRows * (sizeof(float) + sizeof(short)); }
};
__host__ inline size_t tile_stage_bytes(int k) { return (size_t)k * kTileRows * (sizeof(float) + sizeof(short)); }

// One thread issues the two bulk copies of tile `tile` (weights, offsets; the
// operator is stored tile-major) into stage memory `st`; the mbarrier expects
// exactly the bytes issued.
__device__ __forceinline__ void tile_issue(unsigned char *st, uint64_t *bar, int tile, int k, const float *At,
                                           const short *offt)
{
    const TileStage L{k};
    // the stage may have been read by the CTA's threads (generic proxy) before
    // the barrier that precedes this call: order those reads before the
    // copies' writes (async proxy)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(bar, (unsigned)L.bytes());
    const long t0 = (long)tile * k * kTileRows;
    bulk_g2s(st + L.a_off(), At + t0, (unsigned)(k * kTileRows * sizeof(float)), bar);
    bulk_g2s(st + L.o_off(), offt + t0, (unsigned)(k * kTileRows * sizeof(short)), bar);
}

// MODE 0: Chebyshev step (as k_level_v4<0>); MODE 1: residual (as k_level_v4<1>).
// Chunked variant for any k <= kTileMaxK: the row's stencil is read from the
// stage while its gathers run, 8 at a time.
template <int MODE>
__global__ void __launch_bounds__(kTileRows) k_level_tiled(int n, int k, const short *__restrict__ offt,
                                                           const float *__restrict__ At, const float *__restrict__ dinv,
                                                           const uint8_t *__restrict__ btag,
                                                           const float *__restrict__ r, const float *__restrict__ e,
                                                           float *__restrict__ out, float *__restrict__ d, float c1,
                                                           float c2, int first, int *err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int ok_flag;
    const int tid = threadIdx.x;
    const int ntiles = (n + kTileRows - 1) / kTileRows;
    const TileStage L{k};
    const size_t stage = L.bytes();
    unsigned pending = 0;  // bit st: stage st has copies in flight (tracked by thread 0)
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto issue = [&](int tile, int st) {
        if (tid == 0) tile_issue(smem + st * stage, &bar[st], tile, k, At, offt);
        pending |= 1u << st;
    };
    int it = 0;
    if (blockIdx.x < ntiles) issue(blockIdx.x, 0);
    if (blockIdx.x + gridDim.x < ntiles) issue(blockIdx.x + gridDim.x, 1);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
        const int st = it & 1;
        const unsigned parity = (unsigned)((it >> 1) & 1);
        if (tid == 0) ok_flag = mbar_wait_bounded(&bar[st], parity) ? 1 : 0;
        __syncthreads();
        if (!ok_flag) {
            if (tid == 0) {
                atomicOr(err, 1);
                // Best effort before the CTA exits: give the timed-out stage's
                // copies one more bounded spell, then wait (bounded) for the
                // other stage's, so that normally no bulk copy still writes
                // into this CTA's shared memory after it has returned.  The
                // host turns the error flag into MGM_ERR_TIMEOUT.
                mbar_wait_bounded(&bar[st], parity);
                const int o = st ^ 1;
                if (pending & (1u << o)) mbar_wait_bounded(&bar[o], (unsigned)(((it + 1) >> 1) & 1));
            }
            return;
        }
        mbar_try_wait(&bar[st], parity);  // completed: acquires the copied data for this thread
        pending &= ~(1u << st);
        unsigned char *sb = smem + st * stage;
        const int i = tile * kTileRows + tid;
        if (i < n) {
            const float ei = e[i];
            if (btag[i]) {
                out[i] = MODE == 0 ? ei : 0.f;
            } else {
                const float *a = (const float *)(sb + L.a_off()) + tid;
                const short *o = (const short *)(sb + L.o_off()) + tid;
                float s = 0.f;
                int j = 0;
                for (; j + 8 <= k; j += 8) {
                    float av[8], xv[8];
#pragma unroll
                    for (int q = 0; q < 8; q++) {
                        av[q] = a[(j + q) * kTileRows];
                        xv[q] = __ldg(e + i + (int)o[(j + q) * kTileRows]);
                    }
#pragma unroll
                    for (int q = 0; q < 8; q++) s += av[q] * xv[q];
                }
                for (; j < k; j++) s += a[j * kTileRows] * e[i + (int)o[j * kTileRows]];
                if (MODE == 0) {
                    const float q = r[i] - s;
                    const float di = first ? c2 * dinv[i] * q : c1 * d[i] + c2 * dinv[i] * q;
                    d[i] = di;
                    out[i] = ei + di;
                } else {
                    out[i] = r[i] - s;
                }
            }
        }
        __syncthreads();  // every thread is done with stage st
        if (tile + 2 * gridDim.x < ntiles) issue(tile + 2 * gridDim.x, st);
    }
}

// Register variant for k <= 32: a thread copies its row's whole stencil from
// the stage into registers, the CTA syncs, the freed stage starts the copies
// of the tile after next, and the threads issue all k neighbour gathers at
// once (k gathers in flight per row instead of 8).
template <int MODE>
__global__ void __launch_bounds__(kTileRows, 2) k_level_tiled_r(int n, int k, const short *__restrict__ offt,
                                                              const float *__restrict__ At,
                                                              const float *__restrict__ dinv,
                                                              const uint8_t *__restrict__ btag,
                                                              const float *__restrict__ r,
                                                              const float *__restrict__ e, float *__restrict__ out,
                                                              float *__restrict__ d, float c1, float c2, int first,
                                                              int *err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int ok_flag;
    const int tid = threadIdx.x;
    const int ntiles = (n + kTileRows - 1) / kTileRows;
    const TileStage L{k};
    const size_t stage = L.bytes();
    unsigned pending = 0;  // bit st: stage st has copies in flight (tracked by thread 0)
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto issue = [&](int tile, int st) {
        if (tid == 0) tile_issue(smem + st * stage, &bar[st], tile, k, At, offt);
        pending |= 1u << st;
    };
    if (blockIdx.x < ntiles) issue(blockIdx.x, 0);
    if (blockIdx.x + gridDim.x < ntiles) issue(blockIdx.x + gridDim.x, 1);
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
        const int st = it & 1;
        const unsigned parity = (unsigned)((it >> 1) & 1);
        if (tid == 0) ok_flag = mbar_wait_bounded(&bar[st], parity) ? 1 : 0;
        __syncthreads();
        if (!ok_flag) {
            if (tid == 0) {
                atomicOr(err, 1);
                // Best effort before the CTA exits: give the timed-out stage's
                // copies one more bounded spell, then wait (bounded) for the
                // other stage's, so that normally no bulk copy still writes
                // into this CTA's shared memory after it has returned.  The
                // host turns the error flag into MGM_ERR_TIMEOUT.
                mbar_wait_bounded(&bar[st], parity);
                const int o = st ^ 1;
                if (pending & (1u << o)) mbar_wait_bounded(&bar[o], (unsigned)(((it + 1) >> 1) & 1));
            }
            return;
        }
        mbar_try_wait(&bar[st], parity);
        pending &= ~(1u << st);
        const unsigned char *sb = smem + st * stage;
        const float *as = (const float *)(sb + L.a_off());
        const short *os = (const short *)(sb + L.o_off());
        float a[32];
        int o[32];
#pragma unroll
        for (int j = 0; j < 32; j++) {
            a[j] = j < k ? as[j * kTileRows + tid] : 0.f;
            o[j] = j < k ? (int)os[j * kTileRows + tid] : 0;
        }
        __syncthreads();  // stage st is free again
        if (tile + 2 * (int)gridDim.x < ntiles) issue(tile + 2 * gridDim.x, st);
        const int i = tile * kTileRows + tid;
        if (i < n) {
            const float ei = e[i];
            if (btag[i]) {
                out[i] = MODE == 0 ? ei : 0.f;
            } else {
                float x[32];
#pragma unroll
                for (int j = 0; j < 32; j++) x[j] = j < k ? __ldg(e + i + o[j]) : 0.f;
                float s = 0.f;
#pragma unroll
                for (int j = 0; j < 32; j++)
                    if (j < k) s += a[j] * x[j];
                if (MODE == 0) {
                    const float q = r[i] - s;
                    const float di = first ? c2 * dinv[i] * q : c1 * d[i] + c2 * dinv[i] * q;
                    d[i] = di;
                    out[i] = ei + di;
                } else {
                    out[i] = r[i] - s;
                }
            }
        }
    }
}

template <class K>
static int tiled_grid(K kernel, int n, size_t smem)
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        MGM_CUDA(cudaGetDevice(&dev));
        MGM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    int per_sm = 0;
    MGM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTileRows, smem));
    const int tiles = (n + kTileRows - 1) / kTileRows;
    return std::max(1, std::min(tiles, sms * std::max(1, per_sm)));
}

template <int MODE>
static void launch_tiled(const SolveLevel<float> &L, const float *e, float *out, float c1, float c2, int first,
                         cudaStream_t s, Chain &launch)
{
    const size_t smem = 2 * tile_stage_bytes(L.k);
    if (L.k <= 32) {
        MGM_CUDA(cudaFuncSetAttribute(k_level_tiled_r<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(2 * tile_stage_bytes(32))));
        launch.plain(k_level_tiled_r<MODE>, tiled_grid(k_level_tiled_r<MODE>, L.n, smem), kTileRows, smem, s, L.n,
                     L.k, L.offt, L.At, L.dinv, L.btag, L.r, e, out, L.d, c1, c2, first, L.tma_err);
    } else {
        MGM_CUDA(cudaFuncSetAttribute(k_level_tiled<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(2 * tile_stage_bytes(kTileMaxK))));
        launch.plain(k_level_tiled<MODE>, tiled_grid(k_level_tiled<MODE>, L.n, smem), kTileRows, smem, s, L.n, L.k,
                     L.offt, L.At, L.dinv, L.btag, L.r, e, out, L.d, c1, c2, first, L.tma_err);
    }
}

// e = inv * r, one warp per row of the dense coarsest inverse
template <class T, bool COH = false>
__device__ __forceinline__ void dense_row_warp(int w, int lane, int n, const T *__restrict__ inv, const T *r, T *e)
{
    const T *row = inv + (long)w * n;
    T s = T(0);
    for (int j = lane; j < n; j += 32) s += row[j] * ldv<COH>(r + j);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) e[w] = s;
}

template <class T>
__global__ void __launch_bounds__(256) k_dense_solve(int n, const T *__restrict__ inv, const T *__restrict__ r,
                                                     T *__restrict__ e)
{
    pdl_enter();
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    dense_row_warp(warp, lane, n, inv, r, e);
}

// ---------------------------------------------------------------------------
// fused coarse-level V-cycle
//
// The levels below kVecMinRows rows are latency-bound: each operation of the
// V-cycle on them (about 17 per level) is a short kernel whose launch and
// ramp cost as much as its work.  k_coarse_vcycle runs the whole V-cycle from
// level `first` down to the coarsest and back as ONE cooperative launch: one
// CTA per SM, every operation a grid-stride pass over the level's rows with
// the row work of the one-operation kernels (so the same bits), and a grid
// barrier between dependent passes.
// ---------------------------------------------------------------------------
constexpr int kFusedMaxLevels = 8, kFusedMaxCheb = 8, kFusedThreads = 512;

template <class T>
struct FusedLevel {
    int n, ld, k, nb_list, kr, kp;
    const short *off;
    const T *A, *dinv;
    const uint8_t *btag;
    const int *bnd_list, *bnd_idx;
    const T *bnd_A;
    T *r, *e, *e2, *d, *q;
    const short *r_off;   // restriction into this level (compact)
    const int *r_base;
    const T *r_w;
    const short *p_off;   // prolongation from the next coarser level into this one (compact)
    const int *p_base;
    const T *p_w;
    T c1[kFusedMaxCheb], c2[kFusedMaxCheb];  // Chebyshev coefficients of each step
};

template <class T>
struct FusedArgs {
    int first, nl, deg;
    int cn;        // coarsest rows
    const T *cinv; // its dense inverse
    unsigned *bar; // grid barrier: {arrivals, generation}
    int *err;      // set when a barrier wait runs out
    FusedLevel<T> L[kFusedMaxLevels];
};

// Grid barrier of a cooperative launch (all CTAs resident): thread 0 of each
// CTA arrives on a counter; the last arrival resets it and advances the
// generation the others wait on (polled without sleeping: the wait is a few
// microseconds).  The wait is bounded (2^20 polls of L2, under a second);
// when it runs out the CTA records the error and the kernel's CTAs
// return at their next barrier.  Returns false once any CTA has given up.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, int *err, unsigned &gen)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int good = 1;
        __threadfence();
        const unsigned arrived = atomicAdd(&bar[0], 1u) + 1u;
        if (arrived == gridDim.x) {
            atomicExch(&bar[0], 0u);
            __threadfence();
            atomicAdd(&bar[1], 1u);
        } else {
            long spins = 0;
            while (*(volatile unsigned *)&bar[1] == gen) {
                if (++spins > (1L << 20) || ((spins & 255) == 0 && *(volatile int *)err)) {
                    atomicExch(err, 1);
                    good = 0;
                    break;
                }
            }
        }
        __threadfence();
        gen++;
        ok = good && *(volatile int *)err == 0;
    }
    __syncthreads();
    return ok != 0;
}

template <class T>
__global__ void __launch_bounds__(kFusedThreads) k_coarse_vcycle(const __grid_constant__ FusedArgs<T> a)
{
    const int nth = gridDim.x * blockDim.x, tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31, nwarp = nth >> 5, wid = tid >> 5;
    __shared__ T shift;
    unsigned gen = 0;
    if (threadIdx.x == 0) gen = *(volatile unsigned *)&a.bar[1];
#define MGM_SYNC() \
    if (!grid_barrier(a.bar, a.err, gen)) return
    T *cur[kFusedMaxLevels], *nxt[kFusedMaxLevels];
    // one smoothing pass on level l: deg Chebyshev steps, each followed by
    // the boundary rows' exact solve; from e = 0 or from the current e
    auto smooth = [&](int l, bool zero_start) -> bool {
        const FusedLevel<T> &L = a.L[l];
        if (zero_start) {
            for (int i = tid; i < L.n; i += nth) start_row<T, true>(i, L.btag, L.dinv, L.r, cur[l]);
        } else {
            for (int w = wid; w < L.nb_list; w += nwarp)
                bnd_row_warp<T, true>(w, lane, L.bnd_list, L.k, L.bnd_idx, L.bnd_A, L.dinv, L.r, cur[l]);
        }
        if (!grid_barrier(a.bar, a.err, gen)) return false;
        for (int st = 0; st < a.deg; st++) {
            for (int i = tid; i < L.n; i += nth)
                c1_row<0, T, true>(i, L.ld, L.k, L.off, L.A, L.dinv, L.btag, L.r, cur[l], nxt[l], L.d, L.c1[st],
                                   L.c2[st], st == 0 ? 1 : 0);
            if (!grid_barrier(a.bar, a.err, gen)) return false;
            T *t = cur[l]; cur[l] = nxt[l]; nxt[l] = t;
            for (int w = wid; w < L.nb_list; w += nwarp)
                bnd_row_warp<T, true>(w, lane, L.bnd_list, L.k, L.bnd_idx, L.bnd_A, L.dinv, L.r, cur[l]);
            if (!grid_barrier(a.bar, a.err, gen)) return false;
        }
        return true;
    };
    for (int l = a.first; l < a.nl; l++) { cur[l] = a.L[l].e; nxt[l] = a.L[l].e2; }
    for (int l = a.first; l < a.nl - 1; l++) {
        const FusedLevel<T> &L = a.L[l], &C = a.L[l + 1];
        if (!smooth(l, true)) return;
        for (int i = tid; i < L.n; i += nth)
            c1_row<1, T, true>(i, L.ld, L.k, L.off, L.A, L.dinv, L.btag, L.r, cur[l], L.q, L.d, T(0), T(0), 0);
        MGM_SYNC();
        for (int i = tid; i < C.n; i += nth)
            restrict_row<T, true>(i, C.n, C.kr, C.r_off, C.r_base, C.r_w, C.btag, L.q, C.r);
        MGM_SYNC();
    }
    {
        const FusedLevel<T> &L = a.L[a.nl - 1];
        for (int w = wid; w < a.cn; w += nwarp) dense_row_warp<T, true>(w, lane, a.cn, a.cinv, L.r, cur[a.nl - 1]);
        MGM_SYNC();
    }
    for (int l = a.nl - 2; l >= a.first; l--) {
        const FusedLevel<T> &L = a.L[l];
        if (threadIdx.x < 32) {
            const T s = prolong_shift_warp<T, true>(L.n, L.kp, L.p_off, L.p_base, L.p_w, (const T *)cur[l + 1]);
            if (threadIdx.x == 0) shift = s;
        }
        __syncthreads();
        for (int i = tid; i < L.n; i += nth)
            prolong_row<T, true>(i, L.n, L.kp, L.p_off, L.p_base, L.p_w, (const T *)cur[l + 1], cur[l], shift);
        MGM_SYNC();
        if (!smooth(l, false)) return;
    }
#undef MGM_SYNC
}

// Whether levels first..nl-1 can run fused: small (one-row-per-thread)
// compact levels without the tile-streamed or FP16 operator.
template <class T>
static bool fusable(const std::vector<SolveLevel<T>> &Ls, int first, int deg)
{
    const int nl = (int)Ls.size();
    if (first >= nl - 1 || nl > kFusedMaxLevels || deg > kFusedMaxCheb || deg < 1) return false;
    for (int l = first; l < nl; l++) {
        const SolveLevel<T> &L = Ls[l];
        if (l < nl - 1) {
            if (L.n >= kVecMinRows || !L.off || L.At || L.W16 || !L.p_off) return false;
        }
        if (l > first && !L.r_off) return false;
    }
    return true;
}

template <class T>
static void launch_fused(std::vector<SolveLevel<T>> &Ls, const CoarseSolve<T> &cs, int first, int deg, double ratio,
                         cudaStream_t s, const FusedCtl &fc)
{
    FusedArgs<T> a{};
    a.first = first;
    a.nl = (int)Ls.size();
    a.deg = deg;
    a.cn = cs.n;
    a.cinv = cs.inv;
    a.bar = fc.bar;
    a.err = fc.err;
    for (int l = first; l < a.nl; l++) {
        const SolveLevel<T> &S = Ls[l];
        FusedLevel<T> &F = a.L[l];
        F.n = S.n; F.ld = S.ld; F.k = S.k; F.nb_list = S.nb_list; F.kr = S.kr; F.kp = S.kp;
        F.off = S.off; F.A = S.A; F.dinv = S.dinv; F.btag = S.btag;
        F.bnd_list = S.bnd_list; F.bnd_idx = S.bnd_idx; F.bnd_A = S.bnd_A;
        F.r = S.r; F.e = S.e; F.e2 = S.e2; F.d = S.d; F.q = S.q;
        F.r_off = S.r_off; F.r_base = S.r_base; F.r_w = S.r_w;
        F.p_off = S.p_off; F.p_base = S.p_base; F.p_w = S.p_w;
        // the coefficients smooth() passes to the level kernels, step by step
        const double lM = 1.05 * S.lmax, lm = S.lmax / ratio;
        const double th = 0.5 * (lM + lm), de = 0.5 * (lM - lm), sig = th / de;
        double rho = 1.0 / sig;
        for (int st = 0; st < deg; st++) {
            double c1 = 0, c2;
            if (st == 0) c2 = 1.0 / th;
            else {
                const double rn = 1.0 / (2.0 * sig - rho);
                c1 = rn * rho;
                c2 = 2.0 * rn / de;
                rho = rn;
            }
            F.c1[st] = (T)c1;
            F.c2[st] = (T)c2;
        }
    }
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(fc.blocks);
    cfg.blockDim = dim3(kFusedThreads);
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_coarse_vcycle<T>, a);
    if (e != cudaSuccess) throw Error{1, std::string("kernel launch (cooperative): ") + cudaGetErrorString(e)};
    MGM_LAUNCHED();
}

// Self-test of the grid barrier's bounded wait: CTA 1 returns without
// arriving, so CTA 0's wait runs out, sets *err and returns.
__global__ void k_barrier_selftest(unsigned *bar, int *err)
{
    unsigned gen = 0;
    if (threadIdx.x == 0) gen = *(volatile unsigned *)&bar[1];
    if (blockIdx.x == 1) return;
    grid_barrier(bar, err, gen);
}
cudaError_t launch_barrier_selftest(cudaStream_t s, unsigned *bar, int *err)
{
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2);
    cfg.blockDim = dim3(32);
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_barrier_selftest, bar, err);
}

// a cooperative launch of one CTA that does nothing (capture probe)
__global__ void k_coop_probe(int) {}
cudaError_t launch_coop_probe(cudaStream_t s)
{
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(1);
    cfg.blockDim = dim3(32);
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_coop_probe, 0);
}

int fused_vcycle_blocks()
{
    int dev = 0, sms = 0, per32 = 0, per64 = 0;
    MGM_CUDA(cudaGetDevice(&dev));
    MGM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MGM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per32, k_coarse_vcycle<float>, kFusedThreads, 0));
    MGM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per64, k_coarse_vcycle<double>, kFusedThreads, 0));
    MGM_REQUIRE(per32 >= 1 && per64 >= 1, "fused coarse V-cycle: a CTA does not fit on an SM");
    return sms;  // one CTA per SM
}

void SmootherProfile::mark(cudaStream_t s)
{
    if (used >= ev.size()) {
        size_t old = ev.size();
        ev.resize(std::max<size_t>(256, old * 2));
        for (size_t i = old; i < ev.size(); i++) MGM_CUDA(cudaEventCreate(&ev[i]));
    }
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    MGM_CUDA(cudaStreamIsCapturing(s, &st));
    // inside a capture the record must become an event-record node of the graph
    if (st == cudaStreamCaptureStatusActive) MGM_CUDA(cudaEventRecordWithFlags(ev[used++], s, cudaEventRecordExternal));
    else MGM_CUDA(cudaEventRecord(ev[used++], s));
}

void SmootherProfile::harvest()
{
    for (size_t i = 0; i + 1 < used; i += 2) {
        float t = 0;
        MGM_CUDA(cudaEventElapsedTime(&t, ev[i], ev[i + 1]));
        ms += t;
        launches++;
    }
    used = 0;
}

void SmootherProfile::harvest_graph(size_t first, size_t pairs)
{
    for (size_t q = 0; q < pairs; q++) {
        float t = 0;
        MGM_CUDA(cudaEventElapsedTime(&t, ev[first + 2 * q], ev[first + 2 * q + 1]));
        ms += t;
        launches++;
    }
}

SmootherProfile::~SmootherProfile()
{
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
}

template <class T>
static void smooth(SolveLevel<T> &L, int degree, double ratio, bool zero_start, cudaStream_t s,
                   SmootherProfile *prof, Chain &launch)
{
    const double lM = 1.05 * L.lmax, lm = L.lmax / ratio;
    const double th = 0.5 * (lM + lm), de = 0.5 * (lM - lm), sig = th / de;
    double rho = 1.0 / sig;
    const int nb = blocks_for(L.n, 256), nbb = blocks_for((long)L.nb_list * 32, 256);
    if (zero_start)
        launch(k_start_e<T>, nb, 256, 0, s, L.n, L.btag, L.dinv, L.r, L.e);
    else
        launch(k_bnd_exact<T>, nbb, 256, 0, s, L.nb_list, L.bnd_list, L.k, L.bnd_idx, L.bnd_A, L.dinv, L.r, L.e);
    for (int step = 0; step < degree; step++) {
        double c1 = 0, c2;
        if (step == 0) c2 = 1.0 / th;
        else {
            const double rn = 1.0 / (2.0 * sig - rho);
            c1 = rn * rho;
            c2 = 2.0 * rn / de;
            rho = rn;
        }
        if (prof) {
            prof->mark(s);
            launch.broken();
        }
        bool done = false;
        if constexpr (sizeof(T) == 4) {
            if (L.At) {
                launch_tiled<0>(L, L.e, L.e2, (float)c1, (float)c2, step == 0 ? 1 : 0, s, launch);
                done = true;
            }
        }
        if (done) {
        } else if (L.off) {
            launch_compact<0, T>(L, L.e, L.e2, (T)c1, (T)c2, step == 0 ? 1 : 0, s, launch);
        } else {
            launch(k_cheb<T>, nb, 256, 0, s, L.n, L.ld, L.k, L.idx, L.A, L.dinv, L.btag, L.r, L.e, L.e2, L.d, (T)c1,
                   (T)c2, step == 0 ? 1 : 0);
        }
        if (prof) {
            prof->mark(s);
            launch.broken();
        }
        std::swap(L.e, L.e2);
        launch(k_bnd_exact<T>, nbb, 256, 0, s, L.nb_list, L.bnd_list, L.k, L.bnd_idx, L.bnd_A, L.dinv, L.r, L.e);
    }
}

template <class T>
static void vcycle_rec(std::vector<SolveLevel<T>> &Ls, const CoarseSolve<T> &cs, int l, int deg, double ratio,
                       cudaStream_t s, SmootherProfile *prof, Chain &launch, const FusedCtl *fused)
{
    SmootherProfile *lp = (l == 0 && prof && prof->on) ? prof : nullptr;
    SolveLevel<T> &L = Ls[l];
    const int nl = (int)Ls.size();
    if (fused && fused->on && fusable(Ls, l, deg)) {
        // levels l..nl-1 in one cooperative launch; each level's correction
        // ends in its e buffer, as after the 2 deg swaps of the per-level path
        launch_fused(Ls, cs, l, deg, ratio, s, *fused);
        launch.after_kernel = true;
        return;
    }
    if (l == nl - 1) {
        launch(k_dense_solve<T>, blocks_for((long)L.n * 32, 256), 256, 0, s, cs.n, cs.inv, L.r, L.e);
        return;
    }
    smooth(L, deg, ratio, true, s, lp, launch);  // from e = 0
    SolveLevel<T> &C = Ls[l + 1];
    bool tiled = false;
    if constexpr (sizeof(T) == 4) {
        if (L.At) {
            launch_tiled<1>(L, L.e, L.q, 0.f, 0.f, 0, s, launch);
            tiled = true;
        }
    }
    if (tiled) {
    } else if (L.off) {
        launch_compact<1, T>(L, L.e, L.q, T(0), T(0), 0, s, launch);
    } else {
        launch(k_residual<T>, blocks_for(L.n, 256), 256, 0, s, L.n, L.ld, L.k, L.idx, L.A, L.btag, L.r, L.e, L.q);
    }
    if (C.r_off)
        launch(k_restrict_o<T>, blocks_for(C.n, 256), 256, 0, s, C.n, C.kr, C.r_off, C.r_base, C.r_w, C.btag, L.q,
               C.r);
    else
        launch(k_restrict<T>, blocks_for(C.n, 256), 256, 0, s, C.n, C.kr, C.r_idx, C.r_w, C.btag, L.q, C.r);
    vcycle_rec(Ls, cs, l + 1, deg, ratio, s, prof, launch, fused);
    if (L.p_off) {
        launch(k_prolong_o<T>, blocks_for(L.n, 256), 256, 0, s, L.n, L.kp, L.p_off, L.p_base, L.p_w, (const T *)C.e,
               L.e);
    } else {
        launch(k_prolong<T>, blocks_for(L.n, 256), 256, 0, s, L.n, L.kp, L.p_idx, L.p_w, (const T *)C.e, L.e);
    }
    smooth(L, deg, ratio, false, s, lp, launch);
}

template <class T>
void vcycle(std::vector<SolveLevel<T>> &Ls, const CoarseSolve<T> &cs, int cheb_degree, double cheb_ratio,
            cudaStream_t s, SmootherProfile *prof, bool chain, const FusedCtl *fused)
{
    Chain launch;
    launch.enabled = chain;
    vcycle_rec(Ls, cs, 0, cheb_degree, cheb_ratio, s, prof, launch, fused);
}

// Chebyshev smoothing of A e = r on one level from e = 0 (r already in L.r);
// returns the buffer holding e.
template <class T>
const T *smooth_from_zero(SolveLevel<T> &L, int degree, double ratio, cudaStream_t s, bool chain)
{
    Chain launch;
    launch.enabled = chain;
    smooth(L, degree, ratio, true, s, nullptr, launch);  // from e = 0
    return L.e;
}
template const double *smooth_from_zero<double>(SolveLevel<double> &, int, double, cudaStream_t, bool);
template const float *smooth_from_zero<float>(SolveLevel<float> &, int, double, cudaStream_t, bool);

template void vcycle<double>(std::vector<SolveLevel<double>> &, const CoarseSolve<double> &, int, double, cudaStream_t,
                             SmootherProfile *, bool, const FusedCtl *);
template void vcycle<float>(std::vector<SolveLevel<float>> &, const CoarseSolve<float> &, int, double, cudaStream_t,
                            SmootherProfile *, bool, const FusedCtl *);

// ---------------------------------------------------------------------------
// spectral radius of D^-1 A restricted to interior rows (power iteration)
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_power_step(int n, int k, const int *__restrict__ idx, const T *__restrict__ A,
                                                    const T *__restrict__ dinv, const uint8_t *__restrict__ btag,
                                                    const double *__restrict__ v, double *__restrict__ w,
                                                    double *__restrict__ partial)
{
    __shared__ double sm[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double val = 0.0;
    if (i < n && !btag[i]) {
        double s = 0.0;
        for (int j = 0; j < k; j++) {
            const long o = (long)j * n + i;
            s += (double)A[o] * v[idx[o]];
        }
        val = (double)dinv[i] * s;
    }
    if (i < n) w[i] = val;
    double sq = block_sum_d<256>(val * val, sm);
    if (threadIdx.x == 0) partial[blockIdx.x] = sq;
}

__global__ void k_seed_vector(int n, const uint8_t *btag, double *v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // deterministic pseudo-random start vector (integer hash of the index)
    unsigned h = (unsigned)i * 2654435761u;
    h ^= h >> 16; h *= 2246822519u; h ^= h >> 13;
    v[i] = btag[i] ? 0.0 : ((double)(h & 0xffffff) / 16777216.0 - 0.5);
}

__global__ void k_scale(int n, double *v, const double *partial, int nparts)
{
    __shared__ double tot;
    if (threadIdx.x == 0) {
        double s = 0;
        for (int t = 0; t < nparts; t++) s += partial[t];
        tot = s > 0 ? 1.0 / sqrt(s) : 0.0;
    }
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] *= tot;
}

template <class T>
void estimate_lmax(SolveLevel<T> &L, cudaStream_t s)
{
    const int nb = blocks_for(L.n, 256);
    DBuf<double> v(L.n), w(L.n), part(nb);
    std::vector<double> hp(nb);
    k_seed_vector<<<nb, 256, 0, s>>>(L.n, L.btag, v.p);
    MGM_LAUNCHED();
    double lam = 0;
    for (int it = 0; it < 40; it++) {
        // normalise v, apply, measure |w|
        k_power_step<T><<<nb, 256, 0, s>>>(L.n, L.k, L.idx, L.A, L.dinv, L.btag, v.p, w.p, part.p);
        MGM_LAUNCHED();
        part.download(hp.data(), nb, s);
        MGM_CUDA(cudaStreamSynchronize(s));
        double sq = 0;
        for (double x : hp) sq += x;
        // |v| is 1 after the first normalisation
        if (it > 0) lam = sqrt(sq);
        k_scale<<<nb, 256, 0, s>>>(L.n, w.p, part.p, nb);
        MGM_LAUNCHED();
        std::swap(v.p, w.p);
    }
    L.lmax = lam > 0 && std::isfinite(lam) ? lam : 2.0;
}

template void estimate_lmax<double>(SolveLevel<double> &, cudaStream_t);
template void estimate_lmax<float>(SolveLevel<float> &, cudaStream_t);

}  // namespace mgm
