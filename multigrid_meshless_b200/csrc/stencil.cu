// stencil.cu -- memory-bound stencil kernels of the fractional step
// (fractional_step_solver.h:47-275) and the reference-semantics multigrid
// (fractional_step_solver.h:150-246).
//
// All operators are ELL, column-major by stencil slot: W[j*n + i], idx[j*n + i],
// so that consecutive threads (consecutive nodes) read consecutive addresses.
// Sums run over j in ascending order with every product and sum rounded
// separately (MGM_MUL / MGM_ADD), which makes these kernels bit-identical to
// the reference's C loops on the same operator values.
#include "stencil.cuh"

namespace mgm {

template <int BS>
__device__ __forceinline__ double block_sum(double v, double *sm)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < BS / 32 ? sm[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

// ---------------------------------------------------------------------------
// multiply_sparse_matrix_vector_gpu (mat_lib.h:80-89)
__global__ void k_spmv_parity(int n, int k, const double *__restrict__ W, const int *__restrict__ idx,
                              const double *__restrict__ f, double *__restrict__ out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double r = 0.0;
    for (int j = 0; j < k; j++) {
        long o = (long)j * n + i;
        r = MGM_ADD(r, MGM_MUL(W[o], f[idx[o]]));
    }
    out[i] = r;
}

void spmv_parity(int n, int k, const double *W, const int *idx, const double *f, double *out, cudaStream_t s)
{
    if (n <= 0) return;
    k_spmv_parity<<<blocks_for(n, 256), 256, 0, s>>>(n, k, W, idx, f, out);
    MGM_LAUNCHED();
}

// ---------------------------------------------------------------------------
// calculate_intermediate_velocity (fractional_step_solver.h:73-114), fused:
// Dx, Dy, (Dz), lap read once and applied to every velocity component.
template <int DIM>
__global__ void __launch_bounds__(256) k_momentum(StepArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = a.n;
    if (i >= n) return;
    double gx[DIM], gy[DIM], gz[DIM], gl[DIM];
#pragma unroll
    for (int c = 0; c < DIM; c++) { gx[c] = 0.0; gy[c] = 0.0; gz[c] = 0.0; gl[c] = 0.0; }
    const double *vel[3] = {a.u, a.v, a.w};
    // slots in chunks of C: the chunk's indices and weights, then its
    // gathers, are in flight together; each sum still runs in slot order
    constexpr int C = DIM == 2 ? 6 : 3;
    int j = 0;
    for (; j + C <= a.k; j += C) {
        int c[C];
        double wx[C], wy[C], wz[C], wl[C], f[DIM][C];
#pragma unroll
        for (int q = 0; q < C; q++) {
            const long o = (long)(j + q) * n + i;
            c[q] = __ldg(a.idx + o);
            wx[q] = __ldg(a.Dx + o);
            wy[q] = __ldg(a.Dy + o);
            wz[q] = DIM == 3 ? __ldg(a.Dz + o) : 0.0;
            wl[q] = __ldg(a.lap + o);
        }
#pragma unroll
        for (int q = 0; q < C; q++)
#pragma unroll
            for (int d = 0; d < DIM; d++) f[d][q] = __ldg(vel[d] + c[q]);
#pragma unroll
        for (int q = 0; q < C; q++)
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                gx[d] = MGM_ADD(gx[d], MGM_MUL(wx[q], f[d][q]));
                gy[d] = MGM_ADD(gy[d], MGM_MUL(wy[q], f[d][q]));
                if (DIM == 3) gz[d] = MGM_ADD(gz[d], MGM_MUL(wz[q], f[d][q]));
                gl[d] = MGM_ADD(gl[d], MGM_MUL(wl[q], f[d][q]));
            }
    }
    for (; j < a.k; j++) {
        const long o = (long)j * n + i;
        const int c = a.idx[o];
        const double wx = a.Dx[o], wy = a.Dy[o], wl = a.lap[o];
        const double wz = DIM == 3 ? a.Dz[o] : 0.0;
#pragma unroll
        for (int q = 0; q < DIM; q++) {
            const double f = vel[q][c];
            gx[q] = MGM_ADD(gx[q], MGM_MUL(wx, f));
            gy[q] = MGM_ADD(gy[q], MGM_MUL(wy, f));
            if (DIM == 3) gz[q] = MGM_ADD(gz[q], MGM_MUL(wz, f));
            gl[q] = MGM_ADD(gl[q], MGM_MUL(wl, f));
        }
    }
    const double ui = a.u[i], vi = a.v[i], wi = a.w[i];
    double *outs[3] = {a.u_new, a.v_new, a.w_new};
#pragma unroll
    for (int q = 0; q < DIM; q++) {
        // in 2D the reference's dpdz array is never written and stays 0
        const double adv = MGM_ADD(MGM_ADD(MGM_MUL(ui, gx[q]), MGM_MUL(vi, gy[q])), MGM_MUL(wi, DIM == 3 ? gz[q] : 0.0));
        const double rhs = MGM_SUB(adv, MGM_MUL(a.nu, gl[q]));
        outs[q][i] = MGM_SUB(vel[q][i], MGM_MUL(a.dt, rhs));
    }
    if (a.dpdn) a.dpdn[i] = gl[DIM - 1];  // the reference leaves lap(last component) in dpdn
}

// calculate_mass_residual + calculate_boundary_dpdn (fractional_step_solver.h:116-148)
template <int DIM>
__global__ void __launch_bounds__(256) k_divergence(StepArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = a.n;
    if (i >= n) return;
    const bool bnd = a.btag[i] != 0;
    if (bnd) {
        const double dx = MGM_DIV(MGM_MUL(MGM_SUB(a.u_new[i], a.u[i]), a.rho), a.dt);
        const double dy = MGM_DIV(MGM_MUL(MGM_SUB(a.v_new[i], a.v[i]), a.rho), a.dt);
        double dn = MGM_ADD(MGM_MUL(dx, a.nx[i]), MGM_MUL(dy, a.ny[i]));
        if (DIM == 3) {
            const double dz = MGM_DIV(MGM_MUL(MGM_SUB(a.w_new[i], a.w[i]), a.rho), a.dt);
            dn = MGM_ADD(dn, MGM_MUL(dz, a.nz[i]));
        }
        if (a.dpdn) a.dpdn[i] = dn;
        return;  // the boundary source keeps its value (zero): homogeneous Neumann rows
    }
    double sx = 0.0, sy = 0.0, sz = 0.0;
    // slots in chunks of C (as k_momentum); each sum in slot order
    constexpr int C = DIM == 2 ? 6 : 3;
    int j = 0;
    for (; j + C <= a.k; j += C) {
        int c[C];
        double wx[C], wy[C], wz[C], fu[C], fv[C], fw[C];
#pragma unroll
        for (int q = 0; q < C; q++) {
            const long o = (long)(j + q) * n + i;
            c[q] = __ldg(a.idx + o);
            wx[q] = __ldg(a.Dx + o);
            wy[q] = __ldg(a.Dy + o);
            wz[q] = DIM == 3 ? __ldg(a.Dz + o) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < C; q++) {
            fu[q] = __ldg(a.u_new + c[q]);
            fv[q] = __ldg(a.v_new + c[q]);
            fw[q] = DIM == 3 ? __ldg(a.w_new + c[q]) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < C; q++) {
            sx = MGM_ADD(sx, MGM_MUL(wx[q], fu[q]));
            sy = MGM_ADD(sy, MGM_MUL(wy[q], fv[q]));
            if (DIM == 3) sz = MGM_ADD(sz, MGM_MUL(wz[q], fw[q]));
        }
    }
    for (; j < a.k; j++) {
        const long o = (long)j * n + i;
        const int c = a.idx[o];
        sx = MGM_ADD(sx, MGM_MUL(a.Dx[o], a.u_new[c]));
        sy = MGM_ADD(sy, MGM_MUL(a.Dy[o], a.v_new[c]));
        if (DIM == 3) sz = MGM_ADD(sz, MGM_MUL(a.Dz[o], a.w_new[c]));
    }
    a.source[i] = MGM_DIV(MGM_MUL(a.rho, MGM_ADD(MGM_ADD(sx, sy), sz)), a.dt);
}

// update_velocity (fractional_step_solver.h:248-265) fused with the steady
// error partial sums of fractional_step_explicit (:63-69); u_old is the
// velocity at the start of the step (the update leaves boundary rows alone).
// Slots in chunks of C (each sum in slot order); the steady-error sums are
// reduced per warp (partial[global warp], summed by k_finish_steady) with no
// CTA barrier, which let warps that finish early hold the CTA's slot.
template <int DIM>
__global__ void __launch_bounds__(256) k_correct(StepArgs a, double *__restrict__ partial)
{
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = a.n;
    const int i = i0 < n ? i0 : n - 1;  // rows past n compute row n-1 and store nothing
    // the row's own values are loaded before the slot loop, so that their
    // latency overlaps it (loaded after it, they added a memory round trip
    // per thread: 200 against 104 us on a 1M-row benchmark)
    const bool bnd = a.btag[i] != 0;
    const double uo = a.u[i], vo = a.v[i], uw = a.u_new[i], vw = a.v_new[i];
    const double wo = DIM == 3 ? a.w[i] : 0.0, ww = DIM == 3 ? a.w_new[i] : 0.0;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    constexpr int C = DIM == 2 ? 10 : 5;
    int j = 0;
    for (; j + C <= a.k; j += C) {
        int c[C];
        double wx[C], wy[C], wz[C], pc[C];
#pragma unroll
        for (int q = 0; q < C; q++) {
            const long o = (long)(j + q) * n + i;
            c[q] = __ldg(a.idx + o);
            wx[q] = __ldg(a.Dx + o);
            wy[q] = __ldg(a.Dy + o);
            wz[q] = DIM == 3 ? __ldg(a.Dz + o) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < C; q++) pc[q] = __ldg(a.p + c[q]);
#pragma unroll
        for (int q = 0; q < C; q++) {
            sx = MGM_ADD(sx, MGM_MUL(wx[q], pc[q]));
            sy = MGM_ADD(sy, MGM_MUL(wy[q], pc[q]));
            if (DIM == 3) sz = MGM_ADD(sz, MGM_MUL(wz[q], pc[q]));
        }
    }
    for (; j < a.k; j++) {
        const long o = (long)j * n + i;
        const double pc = a.p[a.idx[o]];
        sx = MGM_ADD(sx, MGM_MUL(a.Dx[o], pc));
        sy = MGM_ADD(sy, MGM_MUL(a.Dy[o], pc));
        if (DIM == 3) sz = MGM_ADD(sz, MGM_MUL(a.Dz[o], pc));
    }
    double e = 0.0;
    if (i0 < n && !bnd) {
        const double un = MGM_SUB(uw, MGM_DIV(MGM_MUL(a.dt, sx), a.rho));
        const double vn = MGM_SUB(vw, MGM_DIV(MGM_MUL(a.dt, sy), a.rho));
        const double du = un - uo, dv = vn - vo;
        e = du * du + dv * dv;
        a.u[i] = un;
        a.v[i] = vn;
        if (DIM == 3) {
            const double wn = MGM_SUB(ww, MGM_DIV(MGM_MUL(a.dt, sz), a.rho));
            const double dw = wn - wo;
            e += dw * dw;
            a.w[i] = wn;
        }
    }
    for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
    if ((threadIdx.x & 31) == 0) partial[i0 >> 5] = e;
}

__global__ void k_finish_steady(const double *partial, int nparts, int n, double *out)
{
    __shared__ double sm[32];
    double v = 0.0;
    for (int t = threadIdx.x; t < nparts; t += blockDim.x) v += partial[t];
    v = block_sum<256>(v, sm);
    if (threadIdx.x == 0) *out = sqrt(v / n);
}

// mass-residual diagnostic printed by update_velocity (:266-274)
template <int DIM>
__global__ void __launch_bounds__(256) k_mass_diag(StepArgs a, double *__restrict__ partial)
{
    __shared__ double sm[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (i < a.n) {
        double sx = 0.0, sy = 0.0;
        for (int j = 0; j < a.k; j++) {
            const long o = (long)j * a.n + i;
            const int c = a.idx[o];
            sx = MGM_ADD(sx, MGM_MUL(a.Dx[o], a.u[c]));
            sy = MGM_ADD(sy, MGM_MUL(a.Dy[o], a.v[c]));
        }
        e = MGM_MUL(a.rho, fabs(MGM_ADD(sx, sy)));
    }
    e = block_sum<256>(e, sm);
    if (threadIdx.x == 0) partial[blockIdx.x] = e;
}

__global__ void k_finish_mean(const double *partial, int nparts, int n, double *out)
{
    __shared__ double sm[32];
    double v = 0.0;
    for (int t = threadIdx.x; t < nparts; t += blockDim.x) v += partial[t];
    v = block_sum<256>(v, sm);
    if (threadIdx.x == 0) *out = v / n;
}

void launch_momentum(const StepArgs &a, int dim, cudaStream_t s)
{
    if (dim == 3) k_momentum<3><<<blocks_for(a.n, 256), 256, 0, s>>>(a);
    else k_momentum<2><<<blocks_for(a.n, 256), 256, 0, s>>>(a);
    MGM_LAUNCHED();
}
void launch_divergence(const StepArgs &a, int dim, cudaStream_t s)
{
    if (dim == 3) k_divergence<3><<<blocks_for(a.n, 256), 256, 0, s>>>(a);
    else k_divergence<2><<<blocks_for(a.n, 256), 256, 0, s>>>(a);
    MGM_LAUNCHED();
}
void launch_correct(const StepArgs &a, int dim, double *partial, double *d_err, cudaStream_t s)
{
    const int nb = blocks_for(a.n, 256);
    if (dim == 3) k_correct<3><<<nb, 256, 0, s>>>(a, partial);
    else k_correct<2><<<nb, 256, 0, s>>>(a, partial);
    MGM_LAUNCHED();
    k_finish_steady<<<1, 256, 0, s>>>(partial, nb * 8, a.n, d_err);  // one partial per warp
    MGM_LAUNCHED();
}
void launch_mass_diag(const StepArgs &a, int dim, double *partial, double *d_out, cudaStream_t s)
{
    const int nb = blocks_for(a.n, 256);
    if (dim == 3) k_mass_diag<3><<<nb, 256, 0, s>>>(a, partial);
    else k_mass_diag<2><<<nb, 256, 0, s>>>(a, partial);
    MGM_LAUNCHED();
    k_finish_mean<<<1, 256, 0, s>>>(partial, nb, a.n, d_out);
    MGM_LAUNCHED();
}

// ---------------------------------------------------------------------------
// reference-semantics multigrid (fractional_step_solver.h:150-246)
// relaxation sweep (:171-179) in data-parallel (Jacobi) order: every node is
// updated from the previous sweep's values.
__global__ void __launch_bounds__(256) k_ref_sweep(int n, int k, const int *__restrict__ idx,
                                                   const double *__restrict__ lapP, const double *__restrict__ src,
                                                   const double *__restrict__ pin, double *__restrict__ pout, double w1,
                                                   double w2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double sum = 0.0;
    for (int j = 1; j < k; j++) {
        const long o = (long)j * n + i;
        sum = MGM_ADD(sum, MGM_MUL(lapP[o], pin[idx[o]]));
    }
    pout[i] = MGM_ADD(MGM_MUL(w1, MGM_DIV(MGM_SUB(src[i], sum), lapP[i])), MGM_MUL(w2, pin[i]));
}

// p -= p[0] (:180-183) fused with the all-node residual (:185-191).  TIMPLE
// form (timple_solver.h:265-281): the residual uses lap_Poison (passed as lap)
// on interior rows and is 0 on boundary rows (btag non-null).
__global__ void __launch_bounds__(256) k_ref_shift_residual(int n, int k, const int *__restrict__ idx,
                                                            const double *__restrict__ lap,
                                                            const double *__restrict__ src,
                                                            const double *__restrict__ pin, double *__restrict__ pout,
                                                            double *__restrict__ res, const uint8_t *__restrict__ btag)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double pref = pin[0];
    pout[i] = MGM_SUB(pin[i], pref);
    if (btag && btag[i]) { res[i] = 0.0; return; }
    double r = src[i];
    for (int j = 0; j < k; j++) {
        const long o = (long)j * n + i;
        r = MGM_SUB(r, MGM_MUL(lap[o], MGM_SUB(pin[idx[o]], pref)));
    }
    res[i] = r;
}

// calculate_residuals (:236-246): interior rows only.  TIMPLE form
// (timple_solver.h:285-301, zero_boundary): lap_Poison, boundary rows set to 0.
__global__ void __launch_bounds__(256) k_ref_residual_interior(int n, int k, const int *__restrict__ idx,
                                                               const double *__restrict__ lap,
                                                               const uint8_t *__restrict__ btag,
                                                               const double *__restrict__ src,
                                                               const double *__restrict__ p, double *__restrict__ res,
                                                               int zero_boundary)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (btag[i]) {
        if (zero_boundary) res[i] = 0.0;
        return;
    }
    double sum = 0;
    for (int j = 0; j < k; j++) {
        const long o = (long)j * n + i;
        sum = MGM_ADD(sum, MGM_MUL(lap[o], p[idx[o]]));
    }
    res[i] = MGM_SUB(src[i], sum);
}

// restrict_residuals (:198-212) / the sum of prolongate_corrections (:216-227):
// out[i] (+)= sum_j W[j][i] * in[gidx[j][i]] on rows whose tag is 0; rows
// with a tag are left alone, or set to 0 with zero_tagged (the TIMPLE
// restriction writes every coarse row, timple_solver.h:303-317).
__global__ void __launch_bounds__(256) k_ref_transfer(int n, int k, const int *__restrict__ gidx,
                                                      const double *__restrict__ W, const uint8_t *__restrict__ btag,
                                                      const double *__restrict__ in, double *__restrict__ out,
                                                      int accumulate, int zero_tagged)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (btag[i]) {
        if (zero_tagged) out[i] = 0.0;
        return;
    }
    double r = 0.0;
    for (int j = 0; j < k; j++) {
        const long o = (long)j * n + i;
        r = MGM_ADD(r, MGM_MUL(W[o], in[gidx[o]]));
    }
    out[i] = accumulate ? MGM_ADD(out[i], r) : r;
}

__global__ void k_zero_interior(int n, const uint8_t *__restrict__ btag, double *__restrict__ p)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !btag[i]) p[i] = 0.0;
}

void ref_relaxation(const RefLevel &L, double w1, double w2, int num_relax, cudaStream_t s, RefVariant v)
{
    const int nb = blocks_for(L.n, 256);
    for (int it = 0; it < num_relax; it++) {
        k_ref_sweep<<<nb, 256, 0, s>>>(L.n, L.k, L.idx, L.lapP, L.src, L.p, L.ptmp, w1, w2);
        MGM_LAUNCHED();
        if (v == REF_HEAT) {
            // heat_conduction.h:27-35: the sweep alone (no re-pin, no residual)
            MGM_CUDA(cudaMemcpyAsync(L.p, L.ptmp, sizeof(double) * L.n, cudaMemcpyDeviceToDevice, s));
            continue;
        }
        const bool t = v == REF_TIMPLE;
        k_ref_shift_residual<<<nb, 256, 0, s>>>(L.n, L.k, L.idx, t ? L.lapP : L.lap, L.src, L.ptmp, L.p, L.res,
                                                t ? L.btag : nullptr);
        MGM_LAUNCHED();
    }
}

// the TIMPLE and heat residuals are the same: lap_Poison on interior rows, 0 on
// boundary rows (timple_solver.h:285-301, heat_conduction.h:100-113)
void ref_residual_interior(const RefLevel &L, cudaStream_t s, RefVariant v)
{
    const bool t = v != REF_FS;
    k_ref_residual_interior<<<blocks_for(L.n, 256), 256, 0, s>>>(L.n, L.k, L.idx, t ? L.lapP : L.lap, L.btag,
                                                                 L.src, L.p, L.res, t ? 1 : 0);
    MGM_LAUNCHED();
}

// the TIMPLE and heat restrictions write every coarse row (timple_solver.h:303-317,
// heat_conduction.h:57-75)
void ref_restrict(const RefLevel &F, const RefLevel &C, cudaStream_t s, RefVariant v)
{
    k_ref_transfer<<<blocks_for(C.n, 256), 256, 0, s>>>(C.n, F.k, C.r_idx, C.restr, C.btag, F.res, C.src, 0,
                                                        v != REF_FS ? 1 : 0);
    MGM_LAUNCHED();
}

void ref_prolongate(const RefLevel &F, const RefLevel &C, cudaStream_t s, RefVariant v)
{
    k_ref_transfer<<<blocks_for(F.n, 256), 256, 0, s>>>(F.n, C.k, F.p_idx, F.prol, F.btag, C.p, F.p, 1, 0);
    MGM_LAUNCHED();
    if (v == REF_TIMPLE) {
        // every coarse correction reset (timple_solver.h:333-338)
        MGM_CUDA(cudaMemsetAsync(C.p, 0, sizeof(double) * C.n, s));
    } else {
        // coarse interior corrections reset (fractional_step_solver.h:228-233, heat_conduction.h:92-97)
        k_zero_interior<<<blocks_for(C.n, 256), 256, 0, s>>>(C.n, C.btag, C.p);
        MGM_LAUNCHED();
    }
}

// multigrid_Poisson_solver (fractional_step_solver.h:150-166); the TIMPLE
// variant (timple_solver.h:203-220) and the heat-conduction program's cycle
// (mg_heat_conduction.c:57-71) have the same shape over their own routines
void ref_multigrid(std::vector<RefLevel> &Ls, double w1, double w2, int num_relax, int num_vcycles, cudaStream_t s,
                   RefVariant v)
{
    const int nl = (int)Ls.size();
    for (int cyc = 0; cyc < num_vcycles; cyc++) {
        for (int l = 0; l < nl; l++) {
            ref_relaxation(Ls[l], w1, w2, num_relax, s, v);
            ref_residual_interior(Ls[l], s, v);
            if (l != nl - 1) ref_restrict(Ls[l], Ls[l + 1], s, v);
        }
        for (int l = nl - 1; l > 0; l--) {
            ref_prolongate(Ls[l - 1], Ls[l], s, v);
            if (l != 1) ref_relaxation(Ls[l - 1], w1, w2, num_relax, s, v);
        }
    }
}

}  // namespace mgm
