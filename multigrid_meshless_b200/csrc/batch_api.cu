// batch_api.cu -- C ABI of the batched hierarchies (mgm_batch_* in include/mgm.h).
#include <algorithm>

#include "batch.cuh"

using namespace mgm;

namespace {

template <class F>
int bguard(F &&f)
{
    try {
        f();
        return MGM_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    } catch (const std::bad_alloc &) {
        set_error(MGM_ERR_NOMEM, "host allocation failed");
        return MGM_ERR_NOMEM;
    } catch (const std::exception &e) {
        set_error(MGM_ERR_ARG, e.what());
        return MGM_ERR_ARG;
    }
}

void check_batch(mgm_batch *b)
{
    MGM_REQUIRE(b != nullptr, "null batch context");
    MGM_CUDA(cudaSetDevice(b->device));
}

BLevel &level_of(mgm_batch *b, int lev)
{
    MGM_REQUIRE(lev >= 0 && lev < b->nl, "level out of range");
    return b->L[lev];
}

template <class T>
void maybe_download(const DBuf<T> &d, T *h, size_t count, cudaStream_t s)
{
    if (h && count) d.download(h, count, s);
}

}  // namespace

extern "C" {

mgm_batch *mgm_batch_create(int dim, int phs_degree, int num_levels)
{
    mgm_batch *out = nullptr;
    const int rc = bguard([&] {
        MGM_REQUIRE(dim == 2 || dim == 3, "mgm_batch_create: dim must be 2 or 3");
        MGM_REQUIRE(phs_degree >= 3 && phs_degree % 2 == 1, "mgm_batch_create: phs_degree must be odd and >= 3");
        MGM_REQUIRE(num_levels >= 1 && num_levels <= kBatchMaxLevels, "mgm_batch_create: 1..8 levels");
        auto *b = new mgm_batch();
        b->dim = dim;
        b->phs = phs_degree;
        b->nl = num_levels;
        cudaError_t e = cudaGetDevice(&b->device);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete b;
            throw Error{MGM_ERR_CUDA, std::string("mgm_batch_create: ") + cudaGetErrorString(e)};
        }
        out = b;
    });
    return rc == MGM_OK ? out : nullptr;
}

void mgm_batch_destroy(mgm_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->s) cudaStreamSynchronize(b->s);
    batch_free_solver(b);
    if (b->h_pinned) cudaFreeHost(b->h_pinned);
    for (cudaEvent_t e : b->ev) if (e) cudaEventDestroy(e);
    cudaStream_t s = b->s;
    delete b;
    if (s) cudaStreamDestroy(s);
}

int mgm_batch_set_level(mgm_batch *b, int lev, int n, int nb, const double *x, const double *y, const double *z,
                        const double *nx, const double *ny, const double *nz, const unsigned char *btag,
                        int poly_degree, const int *k_per_node)
{
    return bguard([&] {
        check_batch(b);
        BLevel &L = level_of(b, lev);
        MGM_REQUIRE(n >= 2 && nb >= 0 && nb <= n, "mgm_batch_set_level: bad node counts");
        MGM_REQUIRE(x && y && nx && ny && btag && k_per_node, "mgm_batch_set_level: null input");
        MGM_REQUIRE(b->dim == 2 || (z && nz), "mgm_batch_set_level: 3D needs z and nz");
        MGM_REQUIRE(poly_degree >= 1, "mgm_batch_set_level: poly_degree must be >= 1");
        const int np = monomials(b->dim, poly_degree).np;
        int kmax = 0;
        for (int i = 0; i < n; i++) {
            const int k = k_per_node[i];
            MGM_REQUIRE(k >= 2 && k <= kMaxK && k + np <= kMaxN, "mgm_batch_set_level: stencil size out of range");
            MGM_REQUIRE(k <= n, "mgm_batch_set_level: stencil larger than the level");
            MGM_REQUIRE(i >= nb || k <= n - nb + 1, "mgm_batch_set_level: boundary stencil larger than the interior");
            kmax = std::max(kmax, k);
        }
        for (int i = 0; i < n; i++) MGM_REQUIRE((btag[i] != 0) == (i < nb), "mgm_batch_set_level: boundary nodes must come first");
        std::vector<double> zero(n, 0.0);
        L.n = n; L.nb = nb; L.poly = poly_degree; L.np = np; L.kmax = kmax;
        L.x.upload(x, n, b->s); L.y.upload(y, n, b->s); L.z.upload(z ? z : zero.data(), n, b->s);
        L.nx.upload(nx, n, b->s); L.ny.upload(ny, n, b->s); L.nz.upload(nz ? nz : zero.data(), n, b->s);
        L.btag.upload(btag, n, b->s);
        L.h_kk.assign(k_per_node, k_per_node + n);
        MGM_CUDA(cudaStreamSynchronize(b->s));
        b->setup_done = false;
    });
}

int mgm_batch_setup(mgm_batch *b, int flags)
{
    return bguard([&] {
        check_batch(b);
        batch_free_solver(b);
        batch_setup(b, (flags & MGM_BATCH_AUTOTUNE) != 0);
        MGM_CUDA(cudaStreamSynchronize(b->s));
    });
}

int mgm_batch_weights_report(mgm_batch *b, double *weights_ms, double *tuning_ms, long long *systems, int *tiles,
                             int *smem_bytes, int *ctas_per_sm)
{
    return bguard([&] {
        check_batch(b);
        MGM_REQUIRE(b->setup_done, "mgm_batch_weights_report: call mgm_batch_setup first");
        if (weights_ms) *weights_ms = b->weights_ms;
        if (tuning_ms) *tuning_ms = b->tuning_ms;
        if (systems) *systems = b->systems;
        if (tiles) *tiles = b->tiles;
        if (smem_bytes) *smem_bytes = b->smem_bytes;
        if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
    });
}

int mgm_batch_num_classes(mgm_batch *b, int *count)
{
    return bguard([&] {
        check_batch(b);
        MGM_REQUIRE(count, "null output");
        *count = (int)b->classes.size();
    });
}

int mgm_batch_class(mgm_batch *b, int idx, int *order, long long *systems, int *team_threads, double *us_per_system)
{
    return bguard([&] {
        check_batch(b);
        MGM_REQUIRE(idx >= 0 && idx < (int)b->classes.size(), "class index out of range");
        const BatchClass &c = b->classes[idx];
        if (order) *order = c.N;
        if (systems) *systems = c.count;
        if (team_threads) *team_threads = c.team;
        if (us_per_system) *us_per_system = c.us_per_system;
    });
}

int mgm_batch_level_size(mgm_batch *b, int lev, int *n, int *nb, long long *nnz, long long *r_nnz, long long *p_nnz)
{
    return bguard([&] {
        check_batch(b);
        BLevel &L = level_of(b, lev);
        if (n) *n = L.n;
        if (nb) *nb = L.nb;
        if (nnz) *nnz = L.nnz;
        if (r_nnz) *r_nnz = L.r_nnz;
        if (p_nnz) *p_nnz = L.p_nnz;
    });
}

int mgm_batch_get_level(mgm_batch *b, int lev, double *x, double *y, double *z, double *nx, double *ny, double *nz,
                        unsigned char *btag, int *k_per_node, int *row_ptr, int *col, double *Dx, double *Dy,
                        double *Dz, double *lap, double *lapP)
{
    return bguard([&] {
        check_batch(b);
        MGM_REQUIRE(b->setup_done, "mgm_batch_get_level: call mgm_batch_setup first");
        BLevel &L = level_of(b, lev);
        cudaStream_t s = b->s;
        const size_t n = L.n, nz_ = (size_t)L.nnz;
        maybe_download(L.x, x, n, s); maybe_download(L.y, y, n, s); maybe_download(L.z, z, n, s);
        maybe_download(L.nx, nx, n, s); maybe_download(L.ny, ny, n, s); maybe_download(L.nz, nz, n, s);
        maybe_download(L.btag, btag, n, s);
        maybe_download(L.kk, k_per_node, n, s);
        maybe_download(L.rp, row_ptr, n + 1, s);
        maybe_download(L.col, col, nz_, s);
        maybe_download(L.Dx, Dx, nz_, s); maybe_download(L.Dy, Dy, nz_, s);
        if (b->dim == 3) maybe_download(L.Dz, Dz, nz_, s);
        maybe_download(L.lap, lap, nz_, s); maybe_download(L.lapP, lapP, nz_, s);
        MGM_CUDA(cudaStreamSynchronize(s));
    });
}

int mgm_batch_get_transfer(mgm_batch *b, int lev, int *rpts, int *ppts, int *r_ptr, int *r_col, double *r_w,
                           int *p_ptr, int *p_col, double *p_w)
{
    return bguard([&] {
        check_batch(b);
        MGM_REQUIRE(b->setup_done, "mgm_batch_get_transfer: call mgm_batch_setup first");
        BLevel &L = level_of(b, lev);
        cudaStream_t s = b->s;
        const size_t n = L.n;
        maybe_download(L.rpts, rpts, n, s);
        maybe_download(L.ppts, ppts, n, s);
        if (lev > 0) {
            maybe_download(L.r_rp, r_ptr, n + 1, s);
            maybe_download(L.r_col, r_col, (size_t)L.r_nnz, s);
            maybe_download(L.r_w64, r_w, (size_t)L.r_nnz, s);
        }
        if (lev < b->nl - 1) {
            maybe_download(L.p_rp, p_ptr, n + 1, s);
            maybe_download(L.p_col, p_col, (size_t)L.p_nnz, s);
            maybe_download(L.p_w64, p_w, (size_t)L.p_nnz, s);
        }
        MGM_CUDA(cudaStreamSynchronize(s));
    });
}

int mgm_batch_set_solver(mgm_batch *b, double rel_tol, int restart, int cheb_degree, double cheb_ratio)
{
    return bguard([&] {
        check_batch(b);
        MGM_REQUIRE(rel_tol > 0 && restart >= 1 && restart <= 32 && cheb_degree >= 1 && cheb_ratio > 1,
                    "mgm_batch_set_solver: bad settings");
        b->tol = rel_tol;
        b->restart = restart;
        b->cheb_deg = cheb_degree;
        b->cheb_ratio = cheb_ratio;
    });
}

int mgm_batch_solve(mgm_batch *b, int mode, int nrhs, const double *rhs, double *sol, int *vcycles, double *rel_res,
                    double *solve_ms)
{
    return bguard([&] {
        check_batch(b);
        MGM_REQUIRE(rhs && sol && vcycles && rel_res, "mgm_batch_solve: null argument");
        batch_solve(b, mode, nrhs, rhs, sol, vcycles, rel_res, solve_ms);
    });
}

}  // extern "C"
