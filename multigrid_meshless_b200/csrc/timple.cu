// timple.cu -- the time-implicit (TIMPLE) step of the reference,
// time_implicit_solver (header_files/timple_solver.h:40-410), on the GPU.
//
// Every product, quotient and sum is rounded separately (MGM_*), in the
// reference's order, so that the kernels are bit-identical to the reference's
// C loops run in the same (data-parallel) sweep order.  Operators are ELL
// [k][n]; the level-0 fields are the context's.
#include "ctx.cuh"

namespace mgm {

void poisson_solve(mgm_ctx *c, int mode, bool timple);

namespace {

struct TimpleArgs {
    int n, k;
    const int *idx;
    const double *Dx, *Dy, *Dz, *lap;
    const uint8_t *btag;
    const double *nx, *ny, *nz;
    double *u, *v, *w, *u_new, *v_new, *w_new, *u_old, *v_old, *w_old;
    double *p_old, *pprime, *dpdx, *dpdy, *dpdz, *dpdn, *source;
    double dt, rho, mu, nu, facRe, facdt;
};

// time_implicit_solver's set-up loop (:44-49): u_old = u = u_new, p' = 0
__global__ void k_t_begin(TimpleArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    a.u_old[i] = a.u_new[i]; a.u[i] = a.u_new[i];
    a.v_old[i] = a.v_new[i]; a.v[i] = a.v_new[i];
    a.w_old[i] = a.w_new[i]; a.w[i] = a.w_new[i];
    a.pprime[i] = 0;
}

// the start of each TIMPLE iteration (:51-56): u = u_new, p' = 0
__global__ void k_t_iter(TimpleArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    a.u[i] = a.u_new[i]; a.v[i] = a.v_new[i]; a.w[i] = a.w_new[i];
    a.pprime[i] = 0;
}

// One momentum sweep of calculate_intermediate_velocity_implicit (:88-173) in
// data-parallel order: interior rows from the previous sweep's values (in*),
// boundary rows copied.
template <int DIM>
__global__ void __launch_bounds__(256) k_t_momentum(TimpleArgs a, const double *__restrict__ iu,
                                                    const double *__restrict__ iv, const double *__restrict__ iw,
                                                    double *__restrict__ ou, double *__restrict__ ov,
                                                    double *__restrict__ ow)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = a.n, k = a.k;
    if (i >= n) return;
    if (a.btag[i]) {
        ou[i] = iu[i]; ov[i] = iv[i];
        if (DIM == 3) ow[i] = iw[i];
        return;
    }
    const double *comp_in[3] = {iu, iv, iw};
    double *comp_out[3] = {ou, ov, ow};
    const double *comp_old[3] = {a.u_old, a.v_old, a.w_old};
    const double *grad[3] = {a.dpdx, a.dpdy, a.dpdz};
    const double lap0 = a.lap[i], dx0 = a.Dx[i], dy0 = a.Dy[i];
    const double dz0 = DIM == 3 ? a.Dz[i] : 0.0;
    const double ui = a.u[i], vi = a.v[i], wi = a.w[i];
#pragma unroll
    for (int cidx = 0; cidx < DIM; cidx++) {
        const double *x = comp_in[cidx];
        double temp1 = 0, temp2 = 0, temp3 = 0, temp4 = 0;
        const double advection_x = MGM_MUL(ui, dx0);
        const double advection_y = MGM_MUL(vi, dy0);
        const double diffusion = MGM_MUL(MGM_MUL(-a.facRe, a.mu), lap0);
        double unsteady = MGM_DIV(1., MGM_MUL(a.dt, a.facdt));
        double denom;
        if (cidx < 2) {
            denom = MGM_ADD(MGM_MUL(a.rho, MGM_ADD(MGM_ADD(advection_x, advection_y), unsteady)), diffusion);
            for (int j = 1; j < k; j++) {
                const long o = (long)j * n + i;
                const double xv = x[a.idx[o]];
                temp1 = MGM_ADD(temp1, MGM_MUL(a.Dx[o], xv));
                temp2 = MGM_ADD(temp2, MGM_MUL(a.Dy[o], xv));
                temp4 = MGM_ADD(temp4, MGM_MUL(a.lap[o], xv));
            }
            if (DIM == 3) {
                denom = MGM_ADD(denom, MGM_MUL(MGM_MUL(a.rho, wi), dz0));
                for (int j = 1; j < k; j++) {
                    const long o = (long)j * n + i;
                    temp3 = MGM_ADD(temp3, MGM_MUL(a.Dz[o], x[a.idx[o]]));
                }
            }
        } else {
            const double advection_z = MGM_MUL(wi, dz0);
            denom = MGM_ADD(MGM_MUL(a.rho, MGM_ADD(MGM_ADD(MGM_ADD(advection_x, advection_y), advection_z), unsteady)),
                            diffusion);
            for (int j = 1; j < k; j++) {
                const long o = (long)j * n + i;
                const double xv = x[a.idx[o]];
                temp1 = MGM_ADD(temp1, MGM_MUL(a.Dx[o], xv));
                temp2 = MGM_ADD(temp2, MGM_MUL(a.Dy[o], xv));
                temp3 = MGM_ADD(temp3, MGM_MUL(a.Dz[o], xv));
                temp4 = MGM_ADD(temp4, MGM_MUL(a.lap[o], xv));
            }
        }
        const double advection = MGM_ADD(MGM_ADD(MGM_MUL(ui, temp1), MGM_MUL(vi, temp2)), MGM_MUL(wi, temp3));
        unsteady = MGM_DIV(comp_old[cidx][i], MGM_MUL(a.dt, a.facdt));
        double num = MGM_MUL(a.rho, MGM_SUB(unsteady, advection));
        num = MGM_SUB(num, MGM_MUL(MGM_MUL(MGM_MUL(MGM_SUB(a.facRe, 1.0), a.mu), lap0), x[i]));
        num = MGM_ADD(num, MGM_MUL(a.mu, temp4));
        num = MGM_SUB(num, grad[cidx][i]);
        comp_out[cidx][i] = MGM_DIV(num, denom);
    }
}

// calculate_mass_residual_implicit (:186-197): source from the divergence
// (dpdz is 0 in 2D: never written there, as in the reference)
__global__ void k_t_source(TimpleArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    a.source[i] = a.btag[i] ? 0.0
                            : MGM_DIV(MGM_MUL(a.rho, MGM_ADD(MGM_ADD(a.dpdx[i], a.dpdy[i]), a.dpdz[i])), a.dt);
}

// update_velocity_implicit (:351-363): interior velocities and pressure
template <int DIM>
__global__ void k_t_update(TimpleArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n || a.btag[i]) return;
    a.u_new[i] = MGM_SUB(a.u_new[i], MGM_DIV(MGM_MUL(a.dt, a.dpdx[i]), a.rho));
    a.v_new[i] = MGM_SUB(a.v_new[i], MGM_DIV(MGM_MUL(a.dt, a.dpdy[i]), a.rho));
    if (DIM == 3) a.w_new[i] = MGM_SUB(a.w_new[i], MGM_DIV(MGM_MUL(a.dt, a.dpdz[i]), a.rho));
    a.p_old[i] = MGM_ADD(a.p_old[i], MGM_MUL(1.0, a.pprime[i]));
}

// p_old -= p_old[0] (:364-368): the reference value is taken first
__global__ void k_t_take(const double *p, double *out) { *out = p[0]; }
__global__ void k_t_shift(int n, double *p, const double *pref)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = MGM_SUB(p[i], *pref);
}

// update_boundary_pressure (:371-410).  The velocity terms are assigned, not
// accumulated, inside the stencil loop (:378-392), so only the last stencil
// slot contributes; the pressure of a boundary row reads interior nodes only.
template <int DIM>
__global__ void k_t_bnd_pressure(TimpleArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = a.n, k = a.k;
    if (i >= n || !a.btag[i]) return;
    const double ui = a.u[i], vi = a.v[i], wi = a.w[i];
    double temp1 = 0, temp2 = 0, temp3 = 0;
    {
        const long o = (long)(k - 1) * n + i;
        const int c = a.idx[o];
        const double L = a.lap[o], dx = a.Dx[o], dy = a.Dy[o];
        const double dz = DIM == 3 ? a.Dz[o] : 0.0;
        const double un = a.u_new[c], vn = a.v_new[c];
        temp1 = MGM_MUL(MGM_MUL(a.nu, L), un);
        temp1 = MGM_SUB(temp1, MGM_MUL(MGM_MUL(ui, un), dx));
        temp1 = MGM_SUB(temp1, MGM_MUL(MGM_MUL(vi, un), dy));
        if (DIM == 3) temp1 = MGM_SUB(temp1, MGM_MUL(MGM_MUL(wi, un), dz));
        temp2 = MGM_MUL(MGM_MUL(a.nu, L), vn);
        temp2 = MGM_SUB(temp2, MGM_MUL(MGM_MUL(ui, vn), dx));
        temp2 = MGM_SUB(temp2, MGM_MUL(MGM_MUL(vi, vn), dy));
        if (DIM == 3) temp2 = MGM_SUB(temp2, MGM_MUL(MGM_MUL(wi, vn), dz));
        if (DIM == 3) {
            const double wn = a.w_new[c];
            temp3 = MGM_MUL(MGM_MUL(a.nu, L), wn);
            temp3 = MGM_SUB(temp3, MGM_MUL(MGM_MUL(ui, wn), dx));
            temp3 = MGM_SUB(temp3, MGM_MUL(MGM_MUL(vi, wn), dy));
            temp3 = MGM_SUB(temp3, MGM_MUL(MGM_MUL(wi, wn), dz));
        }
    }
    const double nxi = a.nx[i], nyi = a.ny[i], nzi = a.nz[i];
    const double dpdn =
        MGM_MUL(a.rho, MGM_ADD(MGM_ADD(MGM_MUL(temp1, nxi), MGM_MUL(temp2, nyi)), MGM_MUL(temp3, nzi)));
    a.dpdn[i] = dpdn;
    double sumx = 0, sumy = 0, sumz = 0, Ap = 0.0;
    for (int j = 1; j < k; j++) {
        const long o = (long)j * n + i;
        const double pc = a.p_old[a.idx[o]];
        sumx = MGM_ADD(sumx, MGM_MUL(a.Dx[o], pc));
        sumy = MGM_ADD(sumy, MGM_MUL(a.Dy[o], pc));
        if (DIM == 3) sumz = MGM_ADD(sumz, MGM_MUL(a.Dz[o], pc));
    }
    Ap = MGM_ADD(Ap, MGM_MUL(a.Dx[i], nxi));
    Ap = MGM_ADD(Ap, MGM_MUL(a.Dy[i], nyi));
    if (DIM == 3) Ap = MGM_ADD(Ap, MGM_MUL(a.Dz[i], nzi));
    a.p_old[i] =
        MGM_DIV(MGM_SUB(MGM_SUB(MGM_SUB(dpdn, MGM_MUL(sumx, nxi)), MGM_MUL(sumy, nyi)), MGM_MUL(sumz, nzi)), Ap);
}

// steady-state error partials (:62-67): e += (du^2 + dv^2) [+ dw^2]
template <int DIM>
__global__ void k_t_steady(TimpleArgs a, double *partial)
{
    __shared__ double sm[256];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (i < a.n) {
        const double du = MGM_SUB(a.u_new[i], a.u_old[i]), dv = MGM_SUB(a.v_new[i], a.v_old[i]);
        e = MGM_ADD(MGM_MUL(du, du), MGM_MUL(dv, dv));
        if (DIM == 3) {
            const double dw = MGM_SUB(a.w_new[i], a.w_old[i]);
            e = MGM_ADD(e, MGM_MUL(dw, dw));
        }
    }
    sm[threadIdx.x] = e;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sm[0];
}

__global__ void k_t_steady_finish(const double *partial, int nparts, int n, double *out)
{
    double s = 0.0;
    for (int t = 0; t < nparts; t++) s += partial[t];
    *out = sqrt(s / n);
}

TimpleArgs timple_args(mgm_ctx *c)
{
    Level &L = c->L[0];
    TimpleArgs a{};
    a.n = L.n; a.k = L.k; a.idx = L.idx.p;
    a.Dx = L.Dx.p; a.Dy = L.Dy.p; a.Dz = L.Dz.p; a.lap = L.lap.p;
    a.btag = L.btag.p; a.nx = L.nx.p; a.ny = L.ny.p; a.nz = L.nz.p;
    a.u = c->u.p; a.v = c->v.p; a.w = c->w.p;
    a.u_new = c->u_new.p; a.v_new = c->v_new.p; a.w_new = c->w_new.p;
    a.u_old = c->u_old.p; a.v_old = c->v_old.p; a.w_old = c->w_old.p;
    a.p_old = c->p_old.p; a.pprime = L.p.p; a.dpdx = c->dpdx.p; a.dpdy = c->dpdy.p; a.dpdz = c->dpdz.p;
    a.dpdn = c->dpdn.p; a.source = L.src.p;
    a.dt = c->dt; a.rho = c->rho; a.mu = c->rho / c->Re; a.nu = c->nu; a.facRe = c->facRe; a.facdt = c->facdt;
    return a;
}

}  // namespace

// calculate_intermediate_velocity_implicit (:72-175)
static void timple_momentum(mgm_ctx *c)
{
    cudaStream_t s = c->s;
    Level &L = c->L[0];
    const int n = L.n, k = L.k, dim = c->dim, nb = blocks_for(n, 256);
    TimpleArgs a = timple_args(c);
    spmv_parity(n, k, L.Dx.p, L.idx.p, c->p_old.p, c->dpdx.p, s);
    spmv_parity(n, k, L.Dy.p, L.idx.p, c->p_old.p, c->dpdy.p, s);
    if (dim == 3) spmv_parity(n, k, L.Dz.p, L.idx.p, c->p_old.p, c->dpdz.p, s);
    double *in[3] = {c->u_new.p, c->v_new.p, c->w_new.p}, *out[3] = {c->tu.p, c->tv.p, c->tw.p};
    for (int sw = 0; sw < c->iter_momentum; sw++) {
        if (dim == 3) k_t_momentum<3><<<nb, 256, 0, s>>>(a, in[0], in[1], in[2], out[0], out[1], out[2]);
        else k_t_momentum<2><<<nb, 256, 0, s>>>(a, in[0], in[1], in[2], out[0], out[1], out[2]);
        MGM_LAUNCHED();
        for (int q = 0; q < 3; q++) std::swap(in[q], out[q]);
    }
    if (in[0] != c->u_new.p) {
        double *dst[3] = {c->u_new.p, c->v_new.p, c->w_new.p};
        for (int q = 0; q < dim; q++)
            MGM_CUDA(cudaMemcpyAsync(dst[q], in[q], sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    }
}

// calculate_mass_residual_implicit (:177-201)
static void timple_mass(mgm_ctx *c)
{
    cudaStream_t s = c->s;
    Level &L = c->L[0];
    const int n = L.n, k = L.k;
    spmv_parity(n, k, L.Dx.p, L.idx.p, c->u_new.p, c->dpdx.p, s);
    spmv_parity(n, k, L.Dy.p, L.idx.p, c->v_new.p, c->dpdy.p, s);
    if (c->dim == 3) spmv_parity(n, k, L.Dz.p, L.idx.p, c->w_new.p, c->dpdz.p, s);
    k_t_source<<<blocks_for(n, 256), 256, 0, s>>>(timple_args(c));
    MGM_LAUNCHED();
}

// update_velocity_implicit (:341-369)
static void timple_update(mgm_ctx *c)
{
    cudaStream_t s = c->s;
    Level &L = c->L[0];
    const int n = L.n, k = L.k, nb = blocks_for(n, 256);
    spmv_parity(n, k, L.Dx.p, L.idx.p, L.p.p, c->dpdx.p, s);
    spmv_parity(n, k, L.Dy.p, L.idx.p, L.p.p, c->dpdy.p, s);
    if (c->dim == 3) spmv_parity(n, k, L.Dz.p, L.idx.p, L.p.p, c->dpdz.p, s);
    if (c->dim == 3) k_t_update<3><<<nb, 256, 0, s>>>(timple_args(c));
    else k_t_update<2><<<nb, 256, 0, s>>>(timple_args(c));
    MGM_LAUNCHED();
    k_t_take<<<1, 1, 0, s>>>(c->p_old.p, c->scal.p);
    MGM_LAUNCHED();
    k_t_shift<<<nb, 256, 0, s>>>(n, c->p_old.p, c->scal.p);
    MGM_LAUNCHED();
}

// update_boundary_pressure (:371-410)
static void timple_boundary_pressure(mgm_ctx *c)
{
    const int nb = blocks_for(c->L[0].n, 256);
    if (c->dim == 3) k_t_bnd_pressure<3><<<nb, 256, 0, c->s>>>(timple_args(c));
    else k_t_bnd_pressure<2><<<nb, 256, 0, c->s>>>(timple_args(c));
    MGM_LAUNCHED();
}

// time_implicit_solver (timple_solver.h:40-70)
double timple_step(mgm_ctx *c, int mode)
{
    cudaStream_t s = c->s;
    const int n = c->L[0].n, nb = blocks_for(n, 256);
    TimpleArgs a = timple_args(c);
    k_t_begin<<<nb, 256, 0, s>>>(a);
    MGM_LAUNCHED();
    for (int it = 0; it < c->iter_timple; it++) {
        k_t_iter<<<nb, 256, 0, s>>>(a);
        MGM_LAUNCHED();
        timple_momentum(c);
        timple_mass(c);
        poisson_solve(c, mode, true);  // the pressure-correction equation, on p' (L.p)
        c->vcycles_acc += mode == MGM_MODE_REFERENCE ? c->num_vcycles : c->last_iters;
        timple_update(c);
        timple_boundary_pressure(c);
    }
    if (c->dim == 3) k_t_steady<3><<<nb, 256, 0, s>>>(a, c->partial.p);
    else k_t_steady<2><<<nb, 256, 0, s>>>(a, c->partial.p);
    MGM_LAUNCHED();
    k_t_steady_finish<<<1, 1, 0, s>>>(c->partial.p, nb, n, c->scal.p + 1);
    MGM_LAUNCHED();
    double e = 0;
    MGM_CUDA(cudaMemcpyAsync(&e, c->scal.p + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
    MGM_CUDA(cudaStreamSynchronize(s));
    return e;
}

void timple_part(mgm_ctx *c, int part, int mode)
{
    switch (part) {
    case MGM_TIMPLE_MOMENTUM: timple_momentum(c); break;
    case MGM_TIMPLE_MASS: timple_mass(c); break;
    case MGM_TIMPLE_PRESSURE: poisson_solve(c, mode, true); break;
    case MGM_TIMPLE_UPDATE: timple_update(c); break;
    case MGM_TIMPLE_BOUNDARY_PRESSURE: timple_boundary_pressure(c); break;
    default: throw Error{MGM_ERR_ARG, "mgm_timple_part: unknown part"};
    }
    MGM_CUDA(cudaStreamSynchronize(c->s));
}

}  // namespace mgm

using namespace mgm;

namespace {
template <class F>
int tguard(F &&f)
{
    try {
        f();
        return MGM_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    } catch (const std::exception &e) {
        set_error(MGM_ERR_ARG, e.what());
        return MGM_ERR_ARG;
    }
}
}  // namespace

extern "C" {

int mgm_set_timple(mgm_ctx *c, int iter_timple, int iter_momentum, double facRe, double facdt)
{
    return tguard([&] {
        MGM_REQUIRE(c != nullptr, "null context");
        MGM_CUDA(cudaSetDevice(c->device));
        MGM_REQUIRE(iter_timple >= 1 && iter_momentum >= 1 && facdt > 0, "mgm_set_timple: bad parameters");
        c->iter_timple = iter_timple;
        c->iter_momentum = iter_momentum;
        c->facRe = facRe;
        c->facdt = facdt;
    });
}

int mgm_timple_part(mgm_ctx *c, int part, int mode)
{
    return tguard([&] {
        MGM_REQUIRE(c != nullptr, "null context");
        MGM_CUDA(cudaSetDevice(c->device));
        MGM_REQUIRE(c->setup_done && c->dt > 0, "mgm_timple_part: call mgm_setup and mgm_set_flow first");
        timple_part(c, part, mode);
    });
}

int mgm_timple_run(mgm_ctx *c, int mode, int nsteps, double *step_ms, long long *vcycles, double *steady_err)
{
    return tguard([&] {
        MGM_REQUIRE(c != nullptr, "null context");
        MGM_CUDA(cudaSetDevice(c->device));
        MGM_REQUIRE(c->setup_done && c->dt > 0, "mgm_timple_run: call mgm_setup and mgm_set_flow first");
        MGM_REQUIRE(nsteps >= 0, "mgm_timple_run: nsteps < 0");
        cudaEvent_t ev[2] = {nullptr, nullptr};
        MGM_CUDA(cudaEventCreate(&ev[0]));
        MGM_CUDA(cudaEventCreate(&ev[1]));
        try {
            c->vcycles_acc = 0;
            double e = 0;
            MGM_CUDA(cudaEventRecord(ev[0], c->s));
            for (int t = 0; t < nsteps; t++) e = timple_step(c, mode);
            MGM_CUDA(cudaEventRecord(ev[1], c->s));
            MGM_CUDA(cudaEventSynchronize(ev[1]));
            float ms = 0;
            MGM_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
            if (step_ms) *step_ms = ms;
            if (vcycles) *vcycles = c->vcycles_acc;
            if (steady_err) *steady_err = e;
        } catch (...) {
            cudaEventDestroy(ev[0]);
            cudaEventDestroy(ev[1]);
            throw;
        }
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
    });
}

int mgm_timple_step(mgm_ctx *c, int mode, double *steady_err)
{
    return tguard([&] {
        MGM_REQUIRE(c != nullptr, "null context");
        MGM_CUDA(cudaSetDevice(c->device));
        MGM_REQUIRE(c->setup_done && c->dt > 0, "mgm_timple_step: call mgm_setup and mgm_set_flow first");
        const double e = timple_step(c, mode);
        if (steady_err) *steady_err = e;
    });
}

}  // extern "C"
