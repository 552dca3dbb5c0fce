// krylov.cu -- FP64 vector kernels of the flexible GMRES outer iteration and
// the dense Gauss-Jordan (partial pivoting) used once at set-up for the
// coarsest-level inverse.
#include "krylov.cuh"

namespace mgm {

template <int BS>
__device__ __forceinline__ double bsum(double v, double *sm)
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

// r = b - A x  (A: pinned FP64 operator, ELL), and per-block |r|^2, |b|^2 partials
__global__ void __launch_bounds__(256) k_resid64(int n, int k, const int *__restrict__ idx, const double *__restrict__ A,
                                                 const double *__restrict__ b, const double *__restrict__ x,
                                                 double *__restrict__ r, double *__restrict__ part)
{
    __shared__ double sm[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double rr = 0, bb = 0;
    if (i < n) {
        const double ri = b[i] - ell_row_dot(idx, A, x, n, k, i);
        r[i] = ri;
        rr = ri * ri;
        bb = b[i] * b[i];
    }
    rr = bsum<256>(rr, sm);
    bb = bsum<256>(bb, sm);
    if (threadIdx.x == 0) { part[2 * blockIdx.x] = rr; part[2 * blockIdx.x + 1] = bb; }
}

// w = A z  (z in precision T)
template <class T>
__global__ void __launch_bounds__(256) k_apply64(int n, int k, const int *__restrict__ idx, const double *__restrict__ A,
                                                 const T *__restrict__ z, double *__restrict__ w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    w[i] = ell_row_dot(idx, A, z, n, k, i);
}

// partial dot products h_c = V_c . w for c < cnt; part[c * nblk + blk]
__global__ void __launch_bounds__(256) k_multidot(int n, int cnt, const double *__restrict__ V, long ldv,
                                                  const double *__restrict__ w, double *__restrict__ part)
{
    __shared__ double sm[32];
    for (int c = 0; c < cnt; c++) {
        double s = 0.0;
        const double *vc = V + c * ldv;
        for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
            s = fma(vc[i], w[i], s);
        s = bsum<256>(s, sm);
        if (threadIdx.x == 0) part[(long)c * gridDim.x + blockIdx.x] = s;
    }
}

// out[c] = sum_t part[c * nblk + t]; one block per c
__global__ void k_reduce_parts(const double *__restrict__ part, int nblk, int cnt, double *__restrict__ out)
{
    __shared__ double sm[32];
    const int c = blockIdx.x;
    if (c >= cnt) return;
    double s = 0.0;
    for (int t = threadIdx.x; t < nblk; t += blockDim.x) s += part[(long)c * nblk + t];
    s = bsum<256>(s, sm);
    if (threadIdx.x == 0) out[c] = s;
}

// w -= sum_c h[c] V_c, and per-block partial |w|^2 of the result (grid-stride)
__global__ void __launch_bounds__(256) k_orth_norm(int n, int cnt, const double *__restrict__ V, long ldv,
                                                   const double *__restrict__ h, double *__restrict__ w,
                                                   double *__restrict__ part)
{
    __shared__ double hs[kMaxKrylov + 1];
    __shared__ double sm[32];
    for (int c = threadIdx.x; c < cnt; c += blockDim.x) hs[c] = h[c];
    __syncthreads();
    double acc = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double s = w[i];
        for (int c = 0; c < cnt; c++) s = fma(-hs[c], V[c * ldv + i], s);
        w[i] = s;
        acc = fma(s, s, acc);
    }
    acc = bsum<256>(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// w -= sum_c h[c] V_c
__global__ void __launch_bounds__(256) k_orth_update(int n, int cnt, const double *__restrict__ V, long ldv,
                                                     const double *__restrict__ h, double *__restrict__ w)
{
    __shared__ double hs[kMaxKrylov + 1];
    for (int c = threadIdx.x; c < cnt; c += blockDim.x) hs[c] = h[c];
    __syncthreads();
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = w[i];
    for (int c = 0; c < cnt; c++) s = fma(-hs[c], V[c * ldv + i], s);
    w[i] = s;
}

// out = in * (1 / *nrm) where nrm holds |.|^2 or |.| (is_sq)
__global__ void k_scale_by(int n, const double *__restrict__ in, double *__restrict__ out, const double *__restrict__ nrm,
                           int is_sq)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double d = is_sq ? sqrt(*nrm) : *nrm;
    out[i] = d > 0 ? in[i] / d : 0.0;
}

// x += sum_c y[c] Z_c  (Z in precision T)
template <class T>
__global__ void __launch_bounds__(256) k_combine(int n, int cnt, const T *__restrict__ Z, long ldz,
                                                 const double *__restrict__ y, double *__restrict__ x)
{
    __shared__ double ys[kMaxKrylov + 1];
    for (int c = threadIdx.x; c < cnt; c += blockDim.x) ys[c] = y[c];
    __syncthreads();
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = x[i];
    for (int c = 0; c < cnt; c++) s = fma(ys[c], (double)Z[c * ldz + i], s);
    x[i] = s;
}

template <class T>
__global__ void k_copy_convert(long n, const double *__restrict__ in, T *__restrict__ out)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (T)in[i];
}

template <class T>
__global__ void k_copy_out(long n, const T *__restrict__ in, T *__restrict__ out)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[i];
}

void resid64(int n, int k, const int *idx, const double *A, const double *b, const double *x, double *r, double *part,
             cudaStream_t s)
{
    k_resid64<<<blocks_for(n, 256), 256, 0, s>>>(n, k, idx, A, b, x, r, part);
    MGM_LAUNCHED();
}
template <class T>
void apply64(int n, int k, const int *idx, const double *A, const T *z, double *w, cudaStream_t s)
{
    k_apply64<T><<<blocks_for(n, 256), 256, 0, s>>>(n, k, idx, A, z, w);
    MGM_LAUNCHED();
}
template void apply64<double>(int, int, const int *, const double *, const double *, double *, cudaStream_t);
template void apply64<float>(int, int, const int *, const double *, const float *, double *, cudaStream_t);

int dot_blocks(int n) { return std::max(1, std::min(blocks_for(n, 256), 148 * 4)); }

void multidot(int n, int cnt, const double *V, long ldv, const double *w, double *part, double *out, cudaStream_t s)
{
    const int nb = dot_blocks(n);
    k_multidot<<<nb, 256, 0, s>>>(n, cnt, V, ldv, w, part);
    MGM_LAUNCHED();
    k_reduce_parts<<<cnt, 256, 0, s>>>(part, nb, cnt, out);
    MGM_LAUNCHED();
}
void reduce_parts(const double *part, int nblk, int cnt, double *out, cudaStream_t s)
{
    k_reduce_parts<<<cnt, 256, 0, s>>>(part, nblk, cnt, out);
    MGM_LAUNCHED();
}
void orth_norm(int n, int cnt, const double *V, long ldv, const double *h, double *w, double *part, double *norm2,
               cudaStream_t s)
{
    const int nb = dot_blocks(n);
    k_orth_norm<<<nb, 256, 0, s>>>(n, cnt, V, ldv, h, w, part);
    MGM_LAUNCHED();
    k_reduce_parts<<<1, 256, 0, s>>>(part, nb, 1, norm2);
    MGM_LAUNCHED();
}
void orth_update(int n, int cnt, const double *V, long ldv, const double *h, double *w, cudaStream_t s)
{
    k_orth_update<<<blocks_for(n, 256), 256, 0, s>>>(n, cnt, V, ldv, h, w);
    MGM_LAUNCHED();
}
void scale_by(int n, const double *in, double *out, const double *nrm, int is_sq, cudaStream_t s)
{
    k_scale_by<<<blocks_for(n, 256), 256, 0, s>>>(n, in, out, nrm, is_sq);
    MGM_LAUNCHED();
}
template <class T>
void combine(int n, int cnt, const T *Z, long ldz, const double *y, double *x, cudaStream_t s)
{
    k_combine<T><<<blocks_for(n, 256), 256, 0, s>>>(n, cnt, Z, ldz, y, x);
    MGM_LAUNCHED();
}
template void combine<double>(int, int, const double *, long, const double *, double *, cudaStream_t);
template void combine<float>(int, int, const float *, long, const double *, double *, cudaStream_t);
template <class T>
void copy_convert(long n, const double *in, T *out, cudaStream_t s)
{
    k_copy_convert<T><<<blocks_for(n, 256), 256, 0, s>>>(n, in, out);
    MGM_LAUNCHED();
}
template void copy_convert<double>(long, const double *, double *, cudaStream_t);
template void copy_convert<float>(long, const double *, float *, cudaStream_t);
template <class T>
void copy_out(long n, const T *in, T *out, cudaStream_t s)
{
    k_copy_out<T><<<blocks_for(n, 256), 256, 0, s>>>(n, in, out);
    MGM_LAUNCHED();
}
template void copy_out<double>(long, const double *, double *, cudaStream_t);
template void copy_out<float>(long, const float *, float *, cudaStream_t);

// ---------------------------------------------------------------------------
// device-resident FGMRES control (FgState, krylov.cuh)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void set_cond(cudaGraphConditionalHandle h, int use, int v)
{
    if (use) cudaGraphSetConditional(h, v ? 1u : 0u);
}

__global__ void k_fg_init(FgState *st, int m, int max_total, int max_restarts, double tol)
{
    st->m = m;
    st->max_total = max_total;
    st->max_restarts = max_restarts;
    st->tol = tol;
    st->j = st->j_done = st->total_it = st->restarts = st->vcycles = 0;
    st->reorth = 0;
    st->go_outer = 1;
    st->go_inner = 0;
    st->status = FG_OK;
    st->beta = st->bnorm = 0.0;
    st->relres = 1.0;
    st->alpha = 0.0;
    st->solves_total++;
}

__global__ void k_fg_clear_totals(FgState *st)
{
    st->err_any = 0;
    st->vcycles_total = 0;
    st->cycles_total = 0;
    st->solves_total = 0;
    st->t_ns = 0;
    st->start_log_relres = 0.0;
}

__global__ void k_fg_time_mark(FgState *st, int end)
{
    const unsigned long long t = global_ns();
    if (end) st->t_ns += t - st->t_mark;
    else st->t_mark = t;
}

// Start of a restart cycle: |r|^2, |b|^2 from the residual kernel's per-block
// partials (fixed-order block reduction), the convergence test, and the
// Krylov right-hand side g = beta e_0.
__global__ void __launch_bounds__(256) k_fg_begin(FgState *st, const double *__restrict__ part, int nbres,
                                                  FgHandles hd)
{
    __shared__ double sm[32];
    double rr = 0.0, bb = 0.0;
    for (int t = threadIdx.x; t < nbres; t += blockDim.x) {
        rr += part[2 * t];
        bb += part[2 * t + 1];
    }
    rr = bsum<256>(rr, sm);
    bb = bsum<256>(bb, sm);
    if (threadIdx.x != 0) return;
    const double bnorm = sqrt(bb), beta = sqrt(rr);
    const double relres = bnorm > 0 ? beta / bnorm : 0.0;
    st->bnorm = bnorm;
    st->beta = beta;
    st->relres = relres;
    // the solve's first cycle: the residual its initial guess left
    if (st->restarts == 0 && st->total_it == 0 && relres > 0 && isfinite(relres))
        st->start_log_relres += log10(relres);
    st->j = 0;
    st->j_done = 0;
    int go = 0;
    if (!isfinite(relres)) {
        st->status = FG_NONFINITE;
        st->err_any |= 1;
    } else if (!(bnorm == 0 || relres < st->tol || st->total_it >= st->max_total)) {
        go = 1;
        st->g[0] = beta;
        for (int i = 1; i <= st->m; i++) st->g[i] = 0.0;
    }
    st->go_inner = go;
    // the cycle begun here is the last one when the restart budget is spent
    st->go_outer = go && (st->restarts + 1 <= st->max_restarts);
    if (go) st->restarts++;
    st->cycles_total++;
    set_cond(hd.inner, hd.use, st->go_inner);
    set_cond(hd.outer, hd.use, st->go_outer);
}

// V_0 = r / beta
__global__ void k_fg_scale0(int n, double *__restrict__ V, const FgState *__restrict__ st)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double d = st->beta;
    V[i] = d > 0 ? V[i] / d : 0.0;
}

template <class T>
__global__ void k_fg_load(int n, const double *__restrict__ V, long ld, const FgState *__restrict__ st,
                          T *__restrict__ out)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (T)V[st->j * ld + i];
}

template <class T>
__global__ void k_fg_store(int n, const T *__restrict__ z, T *__restrict__ Z, long ld, const FgState *__restrict__ st)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) Z[st->j * ld + i] = z[i];
}

// V_{j+1} = A Z_j
template <class T>
__global__ void __launch_bounds__(256) k_fg_apply(int n, int k, const int *__restrict__ idx,
                                                  const double *__restrict__ A, const T *__restrict__ Z, long ld,
                                                  const FgState *__restrict__ st, double *__restrict__ V)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = st->j;
    V[(long)(j + 1) * ld + i] = ell_row_dot(idx, A, Z + (long)j * ld, n, k, i);
}

// partial dot products V_c . w (w = V_{j+1}) for c < cnt (pass 0: j+2, pass 1: j+1)
__global__ void __launch_bounds__(256) k_fg_multidot(int n, const double *__restrict__ V, long ld,
                                                     const FgState *__restrict__ st, int pass,
                                                     double *__restrict__ part)
{
    if (pass == 1 && !st->reorth) return;
    __shared__ double sm[32];
    const int j = st->j;
    const int cnt = pass == 0 ? j + 2 : j + 1;
    const double *w = V + (long)(j + 1) * ld;
    for (int c = 0; c < cnt; c++) {
        double s = 0.0;
        const double *vc = V + c * ld;
        for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
            s = fma(vc[i], w[i], s);
        s = bsum<256>(s, sm);
        if (threadIdx.x == 0) part[(long)c * gridDim.x + blockIdx.x] = s;
    }
}

// h[c] (pass 0) or h2[c] (pass 1) = sum_t part[c * nblk + t], one block per c
__global__ void k_fg_reduce_dots(const double *__restrict__ part, int nblk, FgState *__restrict__ st, int pass)
{
    if (pass == 1 && !st->reorth) return;
    __shared__ double sm[32];
    const int cnt = pass == 0 ? st->j + 2 : st->j + 1;
    const int c = blockIdx.x;
    if (c >= cnt) return;
    double s = 0.0;
    for (int t = threadIdx.x; t < nblk; t += blockDim.x) s += part[(long)c * nblk + t];
    s = bsum<256>(s, sm);
    if (threadIdx.x == 0) (pass == 0 ? st->h : st->h2)[c] = s;
}

// w -= sum_{c <= j} h[c] V_c (h2 for pass 1), per-block partial |w|^2
__global__ void __launch_bounds__(256) k_fg_orth(int n, const double *__restrict__ V, long ld,
                                                 const FgState *__restrict__ st, int pass, double *__restrict__ part)
{
    if (pass == 1 && !st->reorth) return;
    __shared__ double hs[kMaxKrylov + 1];
    __shared__ double sm[32];
    const int j = st->j;
    const int cnt = j + 1;
    const double *h = pass == 0 ? st->h : st->h2;
    for (int c = threadIdx.x; c < cnt; c += blockDim.x) hs[c] = h[c];
    __syncthreads();
    double *w = const_cast<double *>(V) + (long)(j + 1) * ld;
    double acc = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        double s = w[i];
        for (int c = 0; c < cnt; c++) s = fma(-hs[c], V[c * ld + i], s);
        w[i] = s;
        acc = fma(s, s, acc);
    }
    acc = bsum<256>(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

__global__ void k_fg_reduce_nrm(const double *__restrict__ part, int nblk, FgState *__restrict__ st, int pass)
{
    if (pass == 1 && !st->reorth) return;
    __shared__ double sm[32];
    double s = 0.0;
    for (int t = threadIdx.x; t < nblk; t += blockDim.x) s += part[t];
    s = bsum<256>(s, sm);
    if (threadIdx.x == 0) st->nrm = s;
}

// Daniel-Gragg-Kaufman-Stewart test: re-orthogonalise when the first pass
// cancelled more than 1 - 1/sqrt(2) of |w|
__global__ void k_fg_dgks(FgState *st)
{
    const int j = st->j;
    for (int i = 0; i <= j; i++) st->h2[i] = 0.0;
    st->reorth = st->nrm < 0.5 * st->h[j + 1];
}

// V_{j+1} /= |w|
__global__ void k_fg_scale_w(int n, double *__restrict__ V, long ld, const FgState *__restrict__ st)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double d = sqrt(st->nrm);
    double *w = V + (long)(st->j + 1) * ld;
    w[i] = d > 0 ? w[i] / d : 0.0;
}

// End of an Arnoldi step: Hessenberg column j, the previous Givens rotations
// applied to it, a new rotation, the updated residual estimate |g_{j+1}| /
// |b|, and the inner loop's condition.
__global__ void k_fg_arnoldi_end(FgState *st, FgHandles hd)
{
    const int j = st->j, m = st->m;
    double *col = st->H + (long)j * (m + 1);
    for (int i = 0; i <= j; i++) col[i] = st->h[i] + st->h2[i];
    col[j + 1] = sqrt(fmax(st->nrm, 0.0));
    for (int i = 0; i < j; i++) {
        const double t0 = st->cs[i] * col[i] + st->sn[i] * col[i + 1];
        col[i + 1] = -st->sn[i] * col[i] + st->cs[i] * col[i + 1];
        col[i] = t0;
    }
    const double a = col[j], b = col[j + 1];
    const double rden = hypot(a, b);
    st->cs[j] = rden > 0 ? a / rden : 1.0;
    st->sn[j] = rden > 0 ? b / rden : 0.0;
    col[j] = rden;
    col[j + 1] = 0.0;
    st->g[j + 1] = -st->sn[j] * st->g[j];
    st->g[j] = st->cs[j] * st->g[j];
    st->total_it++;
    st->vcycles++;
    st->vcycles_total++;
    st->j_done = j + 1;
    const double est = fabs(st->g[j + 1]) / st->bnorm;
    int go = 0;
    if (!isfinite(est)) {
        // no update from this cycle; the outer loop stops (its condition is
        // set by k_fg_solve_y, a kernel of the outer loop's own body)
        st->status = FG_NONFINITE;
        st->err_any |= 1;
        st->go_outer = 0;
        st->j_done = 0;
    } else if (!(est < st->tol) && j + 1 < m) {
        go = 1;
        st->j = j + 1;
    }
    st->go_inner = go;
    set_cond(hd.inner, hd.use, go);
}

// y = H^-1 g (upper triangular, j_done columns); re-asserts the outer loop's
// condition, which an Arnoldi step may have cleared
__global__ void k_fg_solve_y(FgState *st, FgHandles hd)
{
    set_cond(hd.outer, hd.use, st->go_outer);
    const int jd = st->j_done, m = st->m;
    for (int i = jd - 1; i >= 0; i--) {
        double s = st->g[i];
        for (int q = i + 1; q < jd; q++) s -= st->H[(long)q * (m + 1) + i] * st->y[q];
        st->y[i] = s / st->H[(long)i * (m + 1) + i];
    }
}

// x += sum_{c < j_done} y[c] Z_c
template <class T>
__global__ void __launch_bounds__(256) k_fg_combine(int n, const T *__restrict__ Z, long ld,
                                                    const FgState *__restrict__ st, double *__restrict__ x)
{
    __shared__ double ys[kMaxKrylov + 1];
    const int cnt = st->j_done;
    if (cnt == 0) return;
    for (int c = threadIdx.x; c < cnt; c += blockDim.x) ys[c] = st->y[c];
    __syncthreads();
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = x[i];
    for (int c = 0; c < cnt; c++) s = fma(ys[c], (double)Z[c * ld + i], s);
    x[i] = s;
}

__global__ void k_fg_final(FgState *st)
{
    if (st->status == FG_OK && !(st->relres < st->tol) && st->bnorm > 0) {
        st->status = FG_NOT_CONVERGED;
        st->err_any |= 2;
    }
}

__global__ void k_fg_guess(FgState *st, double *ks, int nd)
{
    const double g0 = ks[0], G00 = ks[2];
    double c0 = 0.0, c1 = 0.0;
    auto one = [](double g, double G) {
        const double q = g / G;
        return G > 0 && isfinite(q) ? q : 0.0;
    };
    if (nd == 1) {
        c0 = one(g0, G00);
    } else {
        const double g1 = ks[1], G01 = ks[4], G11 = ks[5];
        const double det = G00 * G11 - G01 * G01;
        if (!(G00 > 0)) {
            c1 = one(g1, G11);
        } else if (!(G11 > 0) || !(det > 1e-12 * G00 * G11)) {
            c0 = one(g0, G00);
        } else {
            c0 = (G11 * g0 - G01 * g1) / det;
            c1 = (G00 * g1 - G01 * g0) / det;
            if (!isfinite(c0) || !isfinite(c1)) { c0 = one(g0, G00); c1 = 0.0; }
        }
    }
    ks[6] = c0;
    ks[7] = c1;
    st->alpha = nd == 1 ? c0 : c1;
}

__global__ void k_set_scalar(double *dst, double v) { *dst = v; }

void fg_init(FgState *st, int m, int max_total, int max_restarts, double tol, cudaStream_t s)
{
    k_fg_init<<<1, 1, 0, s>>>(st, m, max_total, max_restarts, tol);
    MGM_LAUNCHED();
}
void fg_clear_totals(FgState *st, cudaStream_t s)
{
    k_fg_clear_totals<<<1, 1, 0, s>>>(st);
    MGM_LAUNCHED();
}
void fg_time_mark(FgState *st, int end, cudaStream_t s)
{
    k_fg_time_mark<<<1, 1, 0, s>>>(st, end);
    MGM_LAUNCHED();
}
void fg_begin(FgState *st, const double *part, int nbres, FgHandles hd, cudaStream_t s)
{
    k_fg_begin<<<1, 256, 0, s>>>(st, part, nbres, hd);
    MGM_LAUNCHED();
}
void fg_scale0(int n, double *V, const FgState *st, cudaStream_t s)
{
    k_fg_scale0<<<blocks_for(n, 256), 256, 0, s>>>(n, V, st);
    MGM_LAUNCHED();
}
template <class T>
void fg_load(int n, const double *V, long ld, const FgState *st, T *out, cudaStream_t s)
{
    k_fg_load<T><<<blocks_for(n, 256), 256, 0, s>>>(n, V, ld, st, out);
    MGM_LAUNCHED();
}
template void fg_load<double>(int, const double *, long, const FgState *, double *, cudaStream_t);
template void fg_load<float>(int, const double *, long, const FgState *, float *, cudaStream_t);
template <class T>
void fg_store(int n, const T *z, T *Z, long ld, const FgState *st, cudaStream_t s)
{
    k_fg_store<T><<<blocks_for(n, 256), 256, 0, s>>>(n, z, Z, ld, st);
    MGM_LAUNCHED();
}
template void fg_store<double>(int, const double *, double *, long, const FgState *, cudaStream_t);
template void fg_store<float>(int, const float *, float *, long, const FgState *, cudaStream_t);
template <class T>
void fg_apply(int n, int k, const int *idx, const double *A, const T *Z, long ld, const FgState *st, double *V,
              cudaStream_t s)
{
    k_fg_apply<T><<<blocks_for(n, 256), 256, 0, s>>>(n, k, idx, A, Z, ld, st, V);
    MGM_LAUNCHED();
}
template void fg_apply<double>(int, int, const int *, const double *, const double *, long, const FgState *,
                               double *, cudaStream_t);
template void fg_apply<float>(int, int, const int *, const double *, const float *, long, const FgState *, double *,
                              cudaStream_t);
void fg_gram_schmidt(int n, double *V, long ld, FgState *st, int pass, double *part, cudaStream_t s)
{
    const int nb = dot_blocks(n);
    k_fg_multidot<<<nb, 256, 0, s>>>(n, V, ld, st, pass, part);
    MGM_LAUNCHED();
    k_fg_reduce_dots<<<kMaxKrylov + 2, 256, 0, s>>>(part, nb, st, pass);
    MGM_LAUNCHED();
    k_fg_orth<<<nb, 256, 0, s>>>(n, V, ld, st, pass, part);
    MGM_LAUNCHED();
    k_fg_reduce_nrm<<<1, 256, 0, s>>>(part, nb, st, pass);
    MGM_LAUNCHED();
}
void fg_dgks(FgState *st, cudaStream_t s)
{
    k_fg_dgks<<<1, 1, 0, s>>>(st);
    MGM_LAUNCHED();
}
void fg_scale_w(int n, double *V, long ld, const FgState *st, cudaStream_t s)
{
    k_fg_scale_w<<<blocks_for(n, 256), 256, 0, s>>>(n, V, ld, st);
    MGM_LAUNCHED();
}
void fg_arnoldi_end(FgState *st, FgHandles hd, cudaStream_t s)
{
    k_fg_arnoldi_end<<<1, 1, 0, s>>>(st, hd);
    MGM_LAUNCHED();
}
void fg_solve_y(FgState *st, FgHandles hd, cudaStream_t s)
{
    k_fg_solve_y<<<1, 1, 0, s>>>(st, hd);
    MGM_LAUNCHED();
}
template <class T>
void fg_combine(int n, const T *Z, long ld, const FgState *st, double *x, cudaStream_t s)
{
    k_fg_combine<T><<<blocks_for(n, 256), 256, 0, s>>>(n, Z, ld, st, x);
    MGM_LAUNCHED();
}
template void fg_combine<double>(int, const double *, long, const FgState *, double *, cudaStream_t);
template void fg_combine<float>(int, const float *, long, const FgState *, double *, cudaStream_t);
void fg_final(FgState *st, cudaStream_t s)
{
    k_fg_final<<<1, 1, 0, s>>>(st);
    MGM_LAUNCHED();
}
void fg_guess_coefficients(FgState *st, double *ks, int nd, cudaStream_t s)
{
    k_fg_guess<<<1, 1, 0, s>>>(st, ks, nd);
    MGM_LAUNCHED();
}
void set_scalar(double *dst, double v, cudaStream_t s)
{
    k_set_scalar<<<1, 1, 0, s>>>(dst, v);
    MGM_LAUNCHED();
}

// ---------------------------------------------------------------------------
// dense Gauss-Jordan with partial pivoting on [M | I], one matrix, set-up only
// ---------------------------------------------------------------------------
__global__ void k_pivot_search(int n, const double *M, int col, int *piv_row, double *piv_val)
{
    __shared__ double bv[256];
    __shared__ int bi[256];
    double best = -1;
    int br = col;
    for (int r = col + threadIdx.x; r < n; r += blockDim.x) {
        double v = fabs(M[(long)r * 2 * n + col]);
        if (v > best) { best = v; br = r; }
    }
    bv[threadIdx.x] = best;
    bi[threadIdx.x] = br;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            if (bv[threadIdx.x + off] > bv[threadIdx.x] ||
                (bv[threadIdx.x + off] == bv[threadIdx.x] && bi[threadIdx.x + off] < bi[threadIdx.x])) {
                bv[threadIdx.x] = bv[threadIdx.x + off];
                bi[threadIdx.x] = bi[threadIdx.x + off];
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) { *piv_row = bi[0]; *piv_val = M[(long)bi[0] * 2 * n + col]; }
}

__global__ void k_swap_scale(int n, double *M, int col, const int *piv_row, const double *piv_val)
{
    const int pr = *piv_row;
    const double p = *piv_val;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < 2 * n; c += gridDim.x * blockDim.x) {
        double a = M[(long)col * 2 * n + c], b = M[(long)pr * 2 * n + c];
        if (pr != col) M[(long)pr * 2 * n + c] = a;
        M[(long)col * 2 * n + c] = b / p;
    }
}

__global__ void k_eliminate(int n, double *M, int col, double *colbuf)
{
    // colbuf holds column `col` of every row (taken before the update)
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)n * 2 * n) return;
    const int r = (int)(t / (2 * n)), c = (int)(t % (2 * n));
    if (r == col) return;
    const double f = colbuf[r];
    if (f != 0.0) M[t] -= f * M[(long)col * 2 * n + c];
}

__global__ void k_take_col(int n, const double *M, int col, double *colbuf)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) colbuf[r] = M[(long)r * 2 * n + col];
}

__global__ void k_build_aug_dense(int n, int k, const int *idx, const double *A, double *M)
{
    // M = [A_dense | I], A from the ELL operator (duplicates in a row accumulate)
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double *row = M + (long)i * 2 * n;
    for (int c = 0; c < 2 * n; c++) row[c] = (c == n + i) ? 1.0 : 0.0;
    for (int j = 0; j < k; j++) {
        const long o = (long)j * n + i;
        row[idx[o]] += A[o];
    }
}

__global__ void k_extract_inverse(int n, const double *M, double *inv64, float *inv32)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)n * n) return;
    const int r = (int)(t / n), c = (int)(t % n);
    const double v = M[(long)r * 2 * n + n + c];
    inv64[t] = v;
    inv32[t] = (float)v;
}

void dense_inverse(int n, int k, const int *idx, const double *A, double *inv64, float *inv32, cudaStream_t s)
{
    DBuf<double> M((size_t)n * 2 * n), colbuf(n);
    DBuf<int> piv(1);
    DBuf<double> pval(1);
    k_build_aug_dense<<<blocks_for(n, 128), 128, 0, s>>>(n, k, idx, A, M.p);
    MGM_LAUNCHED();
    for (int c = 0; c < n; c++) {
        k_pivot_search<<<1, 256, 0, s>>>(n, M.p, c, piv.p, pval.p);
        MGM_LAUNCHED();
        k_swap_scale<<<blocks_for(2 * n, 256), 256, 0, s>>>(n, M.p, c, piv.p, pval.p);
        MGM_LAUNCHED();
        k_take_col<<<blocks_for(n, 256), 256, 0, s>>>(n, M.p, c, colbuf.p);
        MGM_LAUNCHED();
        k_eliminate<<<blocks_for((long)n * 2 * n, 256), 256, 0, s>>>(n, M.p, c, colbuf.p);
        MGM_LAUNCHED();
    }
    k_extract_inverse<<<blocks_for((long)n * n, 256), 256, 0, s>>>(n, M.p, inv64, inv32);
    MGM_LAUNCHED();
    MGM_CUDA(cudaStreamSynchronize(s));
}

}  // namespace mgm
