// heat.cu -- the reference's heat-conduction program (mg_heat_conduction.c:
// 43-83, with header_files/heat_conduction.h:24-113 and
// init/init_heat_conduction.c:14-67) on the device-resident levels.
//
// The problem: lap_Poison p = f on level 0 with the manufactured source
// f = -8 pi^2 k^2 sin(2 pi k x) sin(2 pi k y) (pi written 3.14, as the
// reference writes it), Dirichlet rows at the boundary nodes with x == 0
// (row = e_i, right-hand side 1) and Neumann rows elsewhere on the boundary
// (right-hand side the manufactured solution's normal derivative).  The
// sources and the Dirichlet rows are set up on the host with libm, as the
// reference's init code does; the time loop runs the program's own V-cycle
// (SOR sweeps alone, lap_Poison residuals with boundary rows 0, every coarse
// row restricted, coarse interior corrections reset) on the GPU, in
// data-parallel sweep order.  set_boundary_rhs, which the reference calls
// before every cycle, only rewrites the same values, so it runs once here.
#include "ctx.cuh"

#include <cmath>

namespace mgm {

void ref_cycles(mgm_ctx *c, RefVariant v, int num_cycles);

namespace {

// Dirichlet rows: lap_Poison[.][i] = e_0 for the listed rows (ELL [k][n])
__global__ void k_dirichlet_rows(int n, int k, int cnt, const int *__restrict__ rows, double *__restrict__ lapP)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cnt * k) return;
    const int r = rows[t / k], j = t % k;
    lapP[(long)j * n + r] = j == 0 ? 1.0 : 0.0;
}

// per-block sums of (a - b)^2 in a fixed order
__global__ void __launch_bounds__(256) k_sq_diff(int n, const double *__restrict__ a, const double *__restrict__ b,
                                                 double *__restrict__ part)
{
    __shared__ double sm[256];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < n) {
        const double d = MGM_SUB(a[i], b[i]);
        v = MGM_MUL(d, d);
    }
    sm[threadIdx.x] = v;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) sm[threadIdx.x] = MGM_ADD(sm[threadIdx.x], sm[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}

__global__ void k_sum_parts(int nparts, const double *__restrict__ part, double *__restrict__ out)
{
    double s = 0.0;
    for (int t = 0; t < nparts; t++) s = MGM_ADD(s, part[t]);
    *out = s;
}

void heat_init(mgm_ctx *c, int wave)
{
    cudaStream_t s = c->s;
    Level &L0 = c->L[0];
    const int n = L0.n;
    std::vector<double> x(n), y(n), nx(n), ny(n), src(n);
    std::vector<uint8_t> bt(n);
    L0.x.download(x.data(), n, s);
    L0.y.download(y.data(), n, s);
    L0.nx.download(nx.data(), n, s);
    L0.ny.download(ny.data(), n, s);
    L0.btag.download(bt.data(), n, s);
    MGM_CUDA(cudaStreamSynchronize(s));
    const int k = wave;
    // initial_conditions (init_heat_conduction.c:30-49); boundary_conditions
    // (:14-28) sets p = 0 where it already is
    for (int i = 0; i < n; i++)
        src[i] = -8 * 3.14 * 3.14 * k * k * std::sin(2 * 3.14 * k * x[i]) * std::sin(2 * 3.14 * k * y[i]);
    // set_boundary_rhs (:51-65)
    std::vector<int> drows;
    for (int i = 0; i < n; i++) {
        if (!bt[i]) continue;
        if (x[i] == 0) {
            src[i] = 1.0;
            drows.push_back(i);
        } else {
            src[i] = 2 * 3.14 * k *
                     (std::sin(2 * 3.14 * k * x[i]) * std::cos(2 * 3.14 * k * y[i]) * ny[i] +
                      std::cos(2 * 3.14 * k * x[i]) * std::sin(2 * 3.14 * k * y[i]) * nx[i]);
        }
    }
    L0.src.upload(src.data(), n, s);
    if (!drows.empty()) {
        DBuf<int> dr(drows.size());
        dr.upload(drows.data(), drows.size(), s);
        k_dirichlet_rows<<<blocks_for((long)drows.size() * L0.k, 256), 256, 0, s>>>(n, L0.k, (int)drows.size(), dr.p,
                                                                                   L0.lapP.p);
        MGM_LAUNCHED();
        MGM_CUDA(cudaStreamSynchronize(s));
    }
    for (int l = 0; l < c->nl; l++) {
        Level &L = c->L[l];
        L.p.zero(s);
        L.res.zero(s);
        if (l > 0) L.src.zero(s);
    }
    MGM_CUDA(cudaStreamSynchronize(s));
    c->heat_wave = wave;
    c->heat_ready = true;
}

// one pass of the time loop (mg_heat_conduction.c:55-77): num_vcycles cycles;
// returns the sum over level 0 of the squared change of p
double heat_step(mgm_ctx *c)
{
    cudaStream_t s = c->s;
    Level &L0 = c->L[0];
    const int n = L0.n, nb = blocks_for(n, 256);
    MGM_CUDA(cudaMemcpyAsync(c->tu.p, L0.p.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    ref_cycles(c, REF_HEAT, c->num_vcycles);
    k_sq_diff<<<nb, 256, 0, s>>>(n, c->tu.p, L0.p.p, c->partial.p);
    MGM_LAUNCHED();
    k_sum_parts<<<1, 1, 0, s>>>(nb, c->partial.p, c->scal.p + 2);
    MGM_LAUNCHED();
    double e = 0;
    MGM_CUDA(cudaMemcpyAsync(&e, c->scal.p + 2, sizeof(double), cudaMemcpyDeviceToHost, s));
    MGM_CUDA(cudaStreamSynchronize(s));
    return e;
}

template <class F>
int hguard(F &&f)
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
}  // namespace mgm

using namespace mgm;

extern "C" {

int mgm_heat_init(mgm_ctx *c, int wave_number)
{
    return hguard([&] {
        MGM_REQUIRE(c != nullptr, "null context");
        MGM_CUDA(cudaSetDevice(c->device));
        MGM_REQUIRE(c->setup_done, "mgm_heat_init: call mgm_setup first");
        MGM_REQUIRE(c->dim == 2, "mgm_heat_init: the heat-conduction program is two-dimensional");
        heat_init(c, wave_number);
    });
}

int mgm_heat_step(mgm_ctx *c, double *steady_err)
{
    return hguard([&] {
        MGM_REQUIRE(c != nullptr, "null context");
        MGM_CUDA(cudaSetDevice(c->device));
        MGM_REQUIRE(c->setup_done && c->heat_ready, "mgm_heat_step: call mgm_heat_init first");
        const double e = heat_step(c);
        if (steady_err) *steady_err = e;
    });
}

}  // extern "C"
