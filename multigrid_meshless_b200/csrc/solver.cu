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
// Exact solve of the boundary rows, one warp per row.  A boundary row couples
// only to itself and interior nodes, so rows can be updated in place.  The
// rows are stored compactly (row-major [nbl][k]) so that a warp reads them
// with coalesced loads.
template <class T>
__global__ void __launch_bounds__(256) k_bnd_exact(int nbl, const int *__restrict__ list, int k,
                                                   const int *__restrict__ bidx, const T *__restrict__ bA,
                                                   const T *__restrict__ dinv, const T *__restrict__ r,
                                                   T *__restrict__ e, int zero_start)
{
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= nbl) return;
    const int i = list[w];
    if (zero_start) {
        if (lane == 0) e[i] = r[i] * dinv[i];
        return;
    }
    T s = T(0);
    for (int j = lane; j < k; j += 32) s += bA[(long)w * k + j] * e[bidx[(long)w * k + j]];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) e[i] = e[i] + (r[i] - s) * dinv[i];
}

// One Chebyshev step on interior rows: q = r - A e, d = c1*d + c2*D^-1 q, e' = e + d.
// Boundary rows copy e.  zero_start: e is zero except on boundary rows.
template <class T>
__global__ void __launch_bounds__(256) k_cheb(int n, int k, const int *__restrict__ idx, const T *__restrict__ A,
                                              const T *__restrict__ dinv, const uint8_t *__restrict__ btag,
                                              const T *__restrict__ r, const T *__restrict__ e, T *__restrict__ eout,
                                              T *__restrict__ d, T c1, T c2, int first)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const T ei = e[i];
    if (btag[i]) { eout[i] = ei; return; }
    const T q = r[i] - ell_row_dot(idx, A, e, n, k, i);
    const T di = first ? c2 * dinv[i] * q : c1 * d[i] + c2 * dinv[i] * q;
    d[i] = di;
    eout[i] = ei + di;
}

// residual on interior rows (boundary rows are solved exactly: 0)
template <class T>
__global__ void __launch_bounds__(256) k_residual(int n, int k, const int *__restrict__ idx, const T *__restrict__ A,
                                                  const uint8_t *__restrict__ btag, const T *__restrict__ r,
                                                  const T *__restrict__ e, T *__restrict__ q)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (btag[i]) { q[i] = T(0); return; }
    q[i] = r[i] - ell_row_dot(idx, A, e, n, k, i);
}

// coarse rhs: r_c[i] = sum_j Rw[j][i] q_f[Ridx[j][i]] on interior coarse rows, 0 elsewhere
template <class T>
__global__ void __launch_bounds__(256) k_restrict(int n, int k, const int *__restrict__ ridx, const T *__restrict__ rw,
                                                  const uint8_t *__restrict__ btag, const T *__restrict__ qf,
                                                  T *__restrict__ rc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (btag[i] || i == 0) { rc[i] = T(0); return; }
    rc[i] = ell_row_dot(ridx, rw, qf, n, k, i);
}

// e_f[i] += (P e_c)[i] - (P e_c)[0]  (the shift keeps the pinned node uncorrected)
template <class T>
__global__ void __launch_bounds__(256) k_prolong(int n, int k, const int *__restrict__ pidx, const T *__restrict__ pw,
                                                 const T *__restrict__ ec, T *__restrict__ ef)
{
    __shared__ T shift;
    if (threadIdx.x == 0) {
        T s = T(0);
        for (int j = 0; j < k; j++) s += pw[(long)j * n] * ec[pidx[(long)j * n]];
        shift = s;
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
template <class X>
__device__ __forceinline__ float ell_row_dot_o(const short *__restrict__ off, const float *__restrict__ A,
                                               const X *__restrict__ x, long n, int k, long i, int base)
{
    float s = 0.f;
    int j = 0;
    for (; j + 8 <= k; j += 8) {
        int c[8];
        float a[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const long o = (long)(j + q) * n + i;
            c[q] = base + (int)__ldg(off + o);
            a[q] = __ldg(A + o);
        }
#pragma unroll
        for (int q = 0; q < 8; q++) s += a[q] * (float)__ldg(x + c[q]);
    }
    for (; j < k; j++) {
        const long o = (long)j * n + i;
        s += A[o] * (float)x[base + (int)off[o]];
    }
    return s;
}

__global__ void __launch_bounds__(256) k_cheb_o(int n, int k, const short *__restrict__ off,
                                                const float *__restrict__ A, const float *__restrict__ dinv,
                                                const uint8_t *__restrict__ btag, const float *__restrict__ r,
                                                const float *__restrict__ e, float *__restrict__ eout,
                                                float *__restrict__ d, float c1, float c2, int first)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float ei = e[i];
    if (btag[i]) { eout[i] = ei; return; }
    const float q = r[i] - ell_row_dot_o(off, A, e, n, k, i, i);
    const float di = first ? c2 * dinv[i] * q : c1 * d[i] + c2 * dinv[i] * q;
    d[i] = di;
    eout[i] = ei + di;
}

__global__ void __launch_bounds__(256) k_residual_o(int n, int k, const short *__restrict__ off,
                                                    const float *__restrict__ A, const uint8_t *__restrict__ btag,
                                                    const float *__restrict__ r, const float *__restrict__ e,
                                                    float *__restrict__ q)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (btag[i]) { q[i] = 0.f; return; }
    q[i] = r[i] - ell_row_dot_o(off, A, e, n, k, i, i);
}

__global__ void __launch_bounds__(256) k_restrict_o(int n, int k, const short *__restrict__ off,
                                                    const int *__restrict__ base, const float *__restrict__ rw,
                                                    const uint8_t *__restrict__ btag, const float *__restrict__ qf,
                                                    float *__restrict__ rc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (btag[i] || i == 0) { rc[i] = 0.f; return; }
    rc[i] = ell_row_dot_o(off, rw, qf, n, k, i, base[i]);
}

__global__ void __launch_bounds__(256) k_prolong_o(int n, int k, const short *__restrict__ off,
                                                   const int *__restrict__ base, const float *__restrict__ pw,
                                                   const float *__restrict__ ec, float *__restrict__ ef)
{
    __shared__ float shift;
    if (threadIdx.x == 0) shift = ell_row_dot_o(off, pw, ec, n, k, 0, base[0]);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ef[i] += ell_row_dot_o(off, pw, ec, n, k, i, base[i]) - shift;
}

// e = inv * r, one warp per row of the dense coarsest inverse
template <class T>
__global__ void __launch_bounds__(256) k_dense_solve(int n, const T *__restrict__ inv, const T *__restrict__ r,
                                                     T *__restrict__ e)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const T *row = inv + (long)warp * n;
    T s = T(0);
    for (int j = lane; j < n; j += 32) s += row[j] * r[j];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) e[warp] = s;
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
                   SmootherProfile *prof)
{
    const double lM = 1.05 * L.lmax, lm = L.lmax / ratio;
    const double th = 0.5 * (lM + lm), de = 0.5 * (lM - lm), sig = th / de;
    double rho = 1.0 / sig;
    const int nb = blocks_for(L.n, 256), nbb = blocks_for((long)L.nb_list * 32, 256);
    k_bnd_exact<T><<<nbb, 256, 0, s>>>(L.nb_list, L.bnd_list, L.k, L.bnd_idx, L.bnd_A, L.dinv, L.r, L.e,
                                       zero_start ? 1 : 0);
    MGM_LAUNCHED();
    if (zero_start) {
        // interior entries of e must be zero before the first step reads them
        // (done by the caller through a memset of e)
    }
    for (int step = 0; step < degree; step++) {
        double c1 = 0, c2;
        if (step == 0) c2 = 1.0 / th;
        else {
            const double rn = 1.0 / (2.0 * sig - rho);
            c1 = rn * rho;
            c2 = 2.0 * rn / de;
            rho = rn;
        }
        if (prof) prof->mark(s);
        if constexpr (sizeof(T) == 4) {
            if (L.off) {
                k_cheb_o<<<nb, 256, 0, s>>>(L.n, L.k, L.off, L.A, L.dinv, L.btag, L.r, L.e, L.e2, L.d, (float)c1,
                                            (float)c2, step == 0 ? 1 : 0);
            } else {
                k_cheb<T><<<nb, 256, 0, s>>>(L.n, L.k, L.idx, L.A, L.dinv, L.btag, L.r, L.e, L.e2, L.d, (T)c1,
                                             (T)c2, step == 0 ? 1 : 0);
            }
        } else {
            k_cheb<T><<<nb, 256, 0, s>>>(L.n, L.k, L.idx, L.A, L.dinv, L.btag, L.r, L.e, L.e2, L.d, (T)c1, (T)c2,
                                         step == 0 ? 1 : 0);
        }
        MGM_LAUNCHED();
        if (prof) prof->mark(s);
        std::swap(L.e, L.e2);
        k_bnd_exact<T><<<nbb, 256, 0, s>>>(L.nb_list, L.bnd_list, L.k, L.bnd_idx, L.bnd_A, L.dinv, L.r, L.e, 0);
        MGM_LAUNCHED();
    }
}

template <class T>
static void vcycle_rec(std::vector<SolveLevel<T>> &Ls, const CoarseSolve<T> &cs, int l, int deg, double ratio,
                       cudaStream_t s, SmootherProfile *prof)
{
    SmootherProfile *lp = (l == 0 && prof && prof->on) ? prof : nullptr;
    SolveLevel<T> &L = Ls[l];
    const int nl = (int)Ls.size();
    if (l == nl - 1) {
        k_dense_solve<T><<<blocks_for((long)L.n * 32, 256), 256, 0, s>>>(cs.n, cs.inv, L.r, L.e);
        MGM_LAUNCHED();
        return;
    }
    MGM_CUDA(cudaMemsetAsync(L.e, 0, sizeof(T) * L.n, s));
    smooth(L, deg, ratio, true, s, lp);
    SolveLevel<T> &C = Ls[l + 1];
    if constexpr (sizeof(T) == 4) {
        if (L.off) k_residual_o<<<blocks_for(L.n, 256), 256, 0, s>>>(L.n, L.k, L.off, L.A, L.btag, L.r, L.e, L.q);
        else k_residual<T><<<blocks_for(L.n, 256), 256, 0, s>>>(L.n, L.k, L.idx, L.A, L.btag, L.r, L.e, L.q);
        MGM_LAUNCHED();
        if (C.r_off) k_restrict_o<<<blocks_for(C.n, 256), 256, 0, s>>>(C.n, C.kr, C.r_off, C.r_base, C.r_w, C.btag, L.q, C.r);
        else k_restrict<T><<<blocks_for(C.n, 256), 256, 0, s>>>(C.n, C.kr, C.r_idx, C.r_w, C.btag, L.q, C.r);
        MGM_LAUNCHED();
    } else {
        k_residual<T><<<blocks_for(L.n, 256), 256, 0, s>>>(L.n, L.k, L.idx, L.A, L.btag, L.r, L.e, L.q);
        MGM_LAUNCHED();
        k_restrict<T><<<blocks_for(C.n, 256), 256, 0, s>>>(C.n, C.kr, C.r_idx, C.r_w, C.btag, L.q, C.r);
        MGM_LAUNCHED();
    }
    vcycle_rec(Ls, cs, l + 1, deg, ratio, s, prof);
    bool poff = false;
    if constexpr (sizeof(T) == 4) poff = L.p_off != nullptr;
    if (poff) {
        if constexpr (sizeof(T) == 4)
            k_prolong_o<<<blocks_for(L.n, 256), 256, 0, s>>>(L.n, L.kp, L.p_off, L.p_base, L.p_w, C.e, L.e);
    } else {
        k_prolong<T><<<blocks_for(L.n, 256), 256, 0, s>>>(L.n, L.kp, L.p_idx, L.p_w, C.e, L.e);
    }
    MGM_LAUNCHED();
    smooth(L, deg, ratio, false, s, lp);
}

template <class T>
void vcycle(std::vector<SolveLevel<T>> &Ls, const CoarseSolve<T> &cs, int cheb_degree, double cheb_ratio,
            cudaStream_t s, SmootherProfile *prof)
{
    vcycle_rec(Ls, cs, 0, cheb_degree, cheb_ratio, s, prof);
}

// Chebyshev smoothing of A e = r on one level from e = 0 (r already in L.r);
// returns the buffer holding e.
template <class T>
const T *smooth_from_zero(SolveLevel<T> &L, int degree, double ratio, cudaStream_t s)
{
    MGM_CUDA(cudaMemsetAsync(L.e, 0, sizeof(T) * L.n, s));
    smooth(L, degree, ratio, true, s, nullptr);
    return L.e;
}
template const double *smooth_from_zero<double>(SolveLevel<double> &, int, double, cudaStream_t);
template const float *smooth_from_zero<float>(SolveLevel<float> &, int, double, cudaStream_t);

template void vcycle<double>(std::vector<SolveLevel<double>> &, const CoarseSolve<double> &, int, double, cudaStream_t,
                             SmootherProfile *);
template void vcycle<float>(std::vector<SolveLevel<float>> &, const CoarseSolve<float> &, int, double, cudaStream_t,
                            SmootherProfile *);

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
