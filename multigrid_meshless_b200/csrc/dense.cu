// dense.cu -- two stand-alone pieces of the reference's weight construction
// behind the C ABI:
//  - matrixInverse_Gauss_Jordan (header_files/mat_lib.h:423-491) for one
//    matrix: one CTA runs the team Gauss-Jordan of weights.cuh (the single
//    bubble pass on column 0, elimination without pivoting, rows scaled last,
//    every product and quotient rounded separately) on an augmented [A | I]
//    in device memory;
//  - create_laplacian_for_Poisson (header_files/rbf.h:382-399): lap_Poison
//    from lap (interior rows) and the boundary rows' normal derivative
//    Dx nx + Dy ny (+ Dz nz), elementwise.
#include "weights.cuh"
#include "mgm.h"

namespace mgm {
namespace {

__global__ void __launch_bounds__(256) k_gj_inverse(int N, const double *__restrict__ A, double *__restrict__ aug,
                                                    int *__restrict__ perm, double *__restrict__ t,
                                                    double *__restrict__ inv)
{
    const Team tm = Team::block();
    const int W2 = 2 * N;
    for (long e = tm.tid; e < (long)N * W2; e += tm.size) {
        const int i = (int)(e / W2), j = (int)(e % W2);
        aug[e] = j < N ? A[(long)i * N + j] : (j - N == i ? 1.0 : 0.0);
    }
    tm.sync();
    gauss_jordan(tm, aug, perm, t, N);
    for (long e = tm.tid; e < (long)N * N; e += tm.size) {
        const int i = (int)(e / N), j = (int)(e % N);
        inv[e] = aug[(long)perm[i] * W2 + N + j];
    }
}

__global__ void k_lap_poisson(int n, int k, int dim, const double *__restrict__ Dx, const double *__restrict__ Dy,
                              const double *__restrict__ Dz, const double *__restrict__ lap,
                              const double *__restrict__ nx, const double *__restrict__ ny,
                              const double *__restrict__ nz, const unsigned char *__restrict__ btag,
                              double *__restrict__ out)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)n * k) return;
    const int i = (int)(e / k);
    if (!btag[i]) {
        out[e] = lap[e];
        return;
    }
    double v = MGM_ADD(MGM_MUL(Dx[e], nx[i]), MGM_MUL(Dy[e], ny[i]));
    if (dim == 3) v = MGM_ADD(v, MGM_MUL(Dz[e], nz[i]));
    out[e] = v;
}

template <class F>
int dguard(F &&f)
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

int mgm_gauss_jordan(int order, const double *A, double *inverse)
{
    return dguard([&] {
        MGM_REQUIRE(order >= 1 && order <= 1024, "mgm_gauss_jordan: order must be in [1, 1024]");
        MGM_REQUIRE(A != nullptr && inverse != nullptr, "mgm_gauss_jordan: null pointer");
        const size_t nn = (size_t)order * order;
        cudaStream_t s = nullptr;
        MGM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            DBuf<double> dA(nn), aug(2 * nn), t(order), dinv(nn);
            DBuf<int> perm(order);
            dA.upload(A, nn, s);
            k_gj_inverse<<<1, 256, 0, s>>>(order, dA.p, aug.p, perm.p, t.p, dinv.p);
            MGM_LAUNCHED();
            dinv.download(inverse, nn, s);
            MGM_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        MGM_CUDA(cudaStreamDestroy(s));
    });
}

int mgm_laplacian_for_poisson(int n, int k, int dim, const double *Dx, const double *Dy, const double *Dz,
                              const double *lap, const double *nx, const double *ny, const double *nz,
                              const unsigned char *btag, double *lapP)
{
    return dguard([&] {
        MGM_REQUIRE(n > 0 && k > 0 && (dim == 2 || dim == 3), "mgm_laplacian_for_poisson: bad sizes");
        MGM_REQUIRE(Dx && Dy && lap && nx && ny && btag && lapP && (dim == 2 || (Dz && nz)),
                    "mgm_laplacian_for_poisson: null pointer");
        const size_t nk = (size_t)n * k;
        cudaStream_t s = nullptr;
        MGM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        try {
            DBuf<double> dx(nk), dy(nk), dz(dim == 3 ? nk : 1), dl(nk), vx(n), vy(n), vz(n), out(nk);
            DBuf<unsigned char> bt(n);
            dx.upload(Dx, nk, s); dy.upload(Dy, nk, s); dl.upload(lap, nk, s);
            vx.upload(nx, n, s); vy.upload(ny, n, s); bt.upload(btag, n, s);
            if (dim == 3) { dz.upload(Dz, nk, s); vz.upload(nz, n, s); }
            k_lap_poisson<<<blocks_for((long)nk, 256), 256, 0, s>>>(n, k, dim, dx.p, dy.p, dz.p, dl.p, vx.p, vy.p, vz.p,
                                                                   bt.p, out.p);
            MGM_LAUNCHED();
            out.download(lapP, nk, s);
            MGM_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            cudaStreamDestroy(s);
            throw;
        }
        MGM_CUDA(cudaStreamDestroy(s));
    });
}

}  // extern "C"
