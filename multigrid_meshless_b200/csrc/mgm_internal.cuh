// mgm_internal.cuh -- shared declarations of the sm_100a kernels and the host runtime.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>
#include <vector>

#include "mgm_math.h"

namespace mgm {

// ---------------------------------------------------------------------------
// error handling: every host entry point converts failures into a status code
// and a thread-local message (mgm_last_error).
// ---------------------------------------------------------------------------
struct Error {
    int code;
    std::string msg;
};
void set_error(int code, const std::string &msg);
extern long long g_launches;

#define MGM_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            throw ::mgm::Error{1, std::string(#call) + ": " + cudaGetErrorString(e_)};              \
    } while (0)

#define MGM_LAUNCHED()                                                                              \
    do {                                                                                            \
        ++::mgm::g_launches;                                                                        \
        cudaError_t e_ = cudaGetLastError();                                                        \
        if (e_ != cudaSuccess)                                                                      \
            throw ::mgm::Error{1, std::string("kernel launch: ") + cudaGetErrorString(e_)};         \
    } while (0)

#define MGM_REQUIRE(cond, msg)                                                                      \
    do {                                                                                            \
        if (!(cond)) throw ::mgm::Error{2, std::string(msg)};                                       \
    } while (0)

constexpr int kMaxPoly = 64;   // monomial table capacity (poly degree <= 6 in 3D)
constexpr int kMaxK = 128;     // stencil width capacity
constexpr int kMaxN = 192;     // k + num_poly_terms capacity of the batched solver

inline int blocks_for(long n, int bs) { return (int)((n + bs - 1) / bs); }

// fused multiply-add a * b + c, rounded once (the contraction the compiler
// applies to s += a * b), spelled out where two kernels must agree bit for bit
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// sum_j A[j][i] * x[idx[j][i]] over an ELL row (column-major by stencil slot).
// Slots are fetched in chunks of 8 (16 independent loads in flight per
// thread, then 8 gathers) to hide DRAM latency; the products are summed in
// slot order.  For kernels that need no particular rounding sequence.
template <class T, class X>
__device__ __forceinline__ T ell_row_dot(const int *__restrict__ idx, const T *__restrict__ A,
                                         const X *__restrict__ x, long n, int k, long i)
{
    T s = T(0);
    int j = 0;
    for (; j + 8 <= k; j += 8) {
        int c[8];
        T a[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
            c[q] = __ldg(idx + (long)(j + q) * n + i);
            a[q] = __ldg(A + (long)(j + q) * n + i);
        }
#pragma unroll
        for (int q = 0; q < 8; q++) s = fma_rn(a[q], (T)__ldg(x + c[q]), s);
    }
    for (; j < k; j++) {
        const long o = (long)j * n + i;
        s = fma_rn(A[o], (T)x[idx[o]], s);
    }
    return s;
}

// device buffer with RAII
template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    DBuf() = default;
    explicit DBuf(size_t count) { alloc(count); }
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    DBuf(DBuf &&o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DBuf &operator=(DBuf &&o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DBuf() { release(); }
    void alloc(size_t count) {
        release();
        n = count;
        if (count) {
            cudaError_t e = cudaMalloc(&p, count * sizeof(T));
            if (e != cudaSuccess) { p = nullptr; n = 0; throw Error{5, std::string("cudaMalloc: ") + cudaGetErrorString(e)}; }
        }
    }
    void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
    void zero(cudaStream_t s) { if (n) { cudaError_t e = cudaMemsetAsync(p, 0, n * sizeof(T), s); if (e != cudaSuccess) throw Error{1, cudaGetErrorString(e)}; } }
    void upload(const T *h, size_t count, cudaStream_t s) {
        if (count > n) alloc(count);
        if (count) MGM_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void download(T *h, size_t count, cudaStream_t s) const {
        if (count) MGM_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
    }
};

// ---------------------------------------------------------------------------
// kernels / launchers (definitions in setup.cu, stencil.cu, solver.cu)
// ---------------------------------------------------------------------------

// exclusive scan of int array (n up to 2^31), returns total through *d_total (device)
void scan_exclusive(const int *d_in, int *d_out, int n, int *d_total, cudaStream_t s);

// kNN: top-k (distance, index) among mask-selected nodes; cloud row-major [nq][k] or
// with self_first: row[0] = q, row[1..k-1] = k-1 nearest.
struct GridIndex {
    int dim = 2, ncx = 1, ncy = 1, ncz = 1;
    double x0 = 0, y0 = 0, z0 = 0, cell = 1;
    DBuf<int> start, items;
};
void grid_build(GridIndex &g, int n, const double *dx, const double *dy, const double *dz,
                const uint8_t *dmask /* nullable: select where mask==0 */, int dim, cudaStream_t s);
// queries: coordinates qx,qy,qz (device) for nq queries; query_ids optional
// mode 0: out[q][0..k-1] = top k; mode 1: out[q][0] = self_id[q], out[q][1..] = top k-1
void knn_query(const GridIndex &g, const double *px, const double *py, const double *pz, int nq,
               const double *qx, const double *qy, const double *qz, const int *self_id, int k, int mode,
               int *out, int ld, cudaStream_t s);

// breadth-first order (rcm_reordering_with_boundarynodes); returns reached count
int bfs_order(int n, int k, const int *d_cloud_rowmajor, int *d_queue1, cudaStream_t s);
void apply_order(int n, int k, const int *d_queue1, double *x, double *y, double *z, double *nx, double *ny,
                 double *nz, uint8_t *btag, int *cloud_rowmajor, cudaStream_t s);
void correct_normals(int n, int k, const double *x, const double *y, const double *z, const uint8_t *btag,
                     const int *cloud_rowmajor, double *nx, double *ny, double *nz, cudaStream_t s);
void avg_dx(int n, int k, int dim, const double *x, const double *y, const double *z, const uint8_t *btag,
            const int *cloud_rowmajor, double *d_out, cudaStream_t s);

// batched saddle-point weights
struct Monomials {
    int np = 0;
    short px[kMaxPoly], py[kMaxPoly], pz[kMaxPoly];
};
Monomials monomials(int dim, int degree);
// derivative weights: outputs row-major [n][k] (Dz nullable in 2D)
void derivative_weights(int n, int k, int dim, int phs, const Monomials &mono, const double *x, const double *y,
                        const double *z, const double *nx, const double *ny, const double *nz, const uint8_t *btag,
                        const int *cloud_rowmajor, double *Dx, double *Dy, double *Dz, double *lap, double *lapP,
                        cudaStream_t s);
// transfer weights: target rows i where (only_interior ? tbtag[i]==0 : i >= rows_from); W row-major [nt][ks]
void transfer_weights(int nt, const double *tx, const double *ty, const double *tz, const uint8_t *tbtag,
                      const int *src_pt, int rows_from, int only_interior, int ks, int dim, int phs,
                      const Monomials &mono, const double *sx, const double *sy, const double *sz,
                      const int *scloud_rowmajor, double *W, cudaStream_t s);

// layout helpers
void transpose_rowmajor_to_ell_d(const double *in, double *out, int n, int k, cudaStream_t s);
void transpose_rowmajor_to_ell_i(const int *in, int *out, int n, int k, cudaStream_t s);
void transpose_ell_to_rowmajor_d(const double *in, double *out, int n, int k, cudaStream_t s);
void transpose_ell_to_rowmajor_i(const int *in, int *out, int n, int k, cudaStream_t s);
void convert_d2f(const double *in, float *out, long n, cudaStream_t s);

// bit-faithful ELL SpMV (mat_lib.h:80-89), cloud/W in ELL [k][n]
void spmv_parity(int n, int k, const double *W, const int *idx, const double *f, double *out, cudaStream_t s);


// kernel launch followed by the launch-error check
template <class... P, class... A>
inline void launch_k(void (*kern)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A... args)
{
    kern<<<grid, block, smem, s>>>(static_cast<P>(args)...);
    MGM_LAUNCHED();
}

// Programmatic dependent launch (griddepcontrol, sm_90 and later).  A kernel
// launched by launch_pdl may have its CTAs scheduled while its predecessor on
// the stream is still finishing; pdl_enter, its first statement, waits until
// the predecessor grid has completed and its memory operations are visible,
// then allows the kernel's own successor to be scheduled early.  Launched
// the ordinary way, pdl_enter returns at once.  Every kernel launched by
// launch_pdl calls pdl_enter before it reads or writes any buffer.
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <class... P, class... A>
inline void launch_pdl(void (*kern)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A... args)
{
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, static_cast<P>(args)...);
    if (e != cudaSuccess) throw Error{1, std::string("kernel launch (programmatic): ") + cudaGetErrorString(e)};
    MGM_LAUNCHED();
}

// The launches of one V-cycle or smoothing pass.  With chaining enabled,
// a kernel whose predecessor on the stream is a kernel of the same chain is
// launched by launch_pdl (such kernels begin with pdl_enter); the first
// launch of a chain, and a launch after an event record (broken()), is an
// ordinary launch.
struct Chain {
    bool enabled = false;
    bool after_kernel = false;
    template <class... P, class... A>
    void operator()(void (*kern)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A... args)
    {
        if (enabled && after_kernel) launch_pdl(kern, grid, block, smem, s, args...);
        else launch_k(kern, grid, block, smem, s, args...);
        after_kernel = true;
    }
    // an ordinary launch of a kernel without pdl_enter inside the chain
    template <class... P, class... A>
    void plain(void (*kern)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A... args)
    {
        launch_k(kern, grid, block, smem, s, args...);
        after_kernel = true;
    }
    void broken() { after_kernel = false; }
};

}  // namespace mgm
