// mgm_api.cu -- host runtime and C ABI (include/mgm.h).
//
// The context owns every device array of every level: the reference's
// jagged host rows (structures.h:44-106) become, per level, SoA coordinates,
// a uint8 boundary tag, and ELL operators column-major by stencil slot.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "ctx.cuh"

namespace mgm {

long long g_launches = 0;
static thread_local std::string t_err;
void set_error(int code, const std::string &msg)
{
    (void)code;
    t_err = msg;
}

}  // namespace mgm

using namespace mgm;

// ---------------------------------------------------------------------------
namespace {

template <class F>
int guard(F &&f)
{
    try {
        f();
        return MGM_OK;
    } catch (const Error &e) {
        t_err = e.msg;
        return e.code;
    } catch (const std::bad_alloc &) {
        t_err = "host allocation failed";
        return MGM_ERR_NOMEM;
    } catch (const std::exception &e) {
        t_err = e.what();
        return MGM_ERR_ARG;
    }
}

cudaStream_t tmp_stream()
{
    static thread_local cudaStream_t s = nullptr;
    if (!s) MGM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    return s;
}

void check_ctx(mgm_ctx *c)
{
    MGM_REQUIRE(c != nullptr, "null context");
    MGM_CUDA(cudaSetDevice(c->device));
}

__global__ void k_gather_idx(int n, int k, const int *__restrict__ pts, const int *__restrict__ src_cloud,
                             int *__restrict__ out)
{
    // out[j][i] = src_cloud[pts[i]][j]
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)n * k) return;
    const int j = (int)(t / n), i = (int)(t % n);
    out[t] = src_cloud[(long)pts[i] * k + j];
}

__global__ void k_pin_operator(int n, int k, const double *__restrict__ lapP, double *__restrict__ A64,
                               double *__restrict__ d64, float *__restrict__ d32)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)n * k) return;
    const int j = (int)(t / n), i = (int)(t % n);
    double a = lapP[t];
    if (i == 0) a = (j == 0) ? 1.0 : 0.0;  // pinned row p[0] = 0
    A64[t] = a;
    if (j == 0) { d64[i] = 1.0 / a; d32[i] = (float)(1.0 / a); }
}

__global__ void k_bc(int n, int kind, const double *x, const double *y, double *u, double *v, double *un, double *vn)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (kind == MGM_BC_LID) {
        if (fabs(y[i] - 1.0) < 1e-9) { u[i] = 1.0; v[i] = 0.0; }
    } else {
        // init_TC.c:37: every product and sum rounded separately, as in the C build
        const double r = sqrt(MGM_ADD(MGM_MUL(x[i], x[i]), MGM_MUL(y[i], y[i])));
        if (fabs(r - 0.5) < 1e-9) {
            u[i] = -y[i] / r; v[i] = x[i] / r;
            un[i] = u[i]; vn[i] = v[i];
        }
    }
}

__global__ void k_zero_pinned(double *b) { b[0] = 0.0; }

// Compatible right-hand sides.  lap_Poison (interior Laplacian rows, Neumann
// boundary rows) is singular with a left null vector z; the pinned solve
// (row 0 replaced by p[0] = 0) puts the part of b along z into row 0, where
// it shows as the residual of the unpinned row-0 equation,
// rho0(x) = x[0] - (lap_Poison p)[0] = z.x / z[0].  Projecting b to
// b - alpha w (w: 1 on interior rows) with alpha = z.b / z.w = rho0(b) / rho0(w)
// makes the system consistent; by linearity its pinned solution is
// p_b - alpha p_w, p_w the pinned solution for w.

// w: 1 on interior rows, 0 on boundary rows
__global__ void k_interior_indicator(int n, const uint8_t *__restrict__ btag, double *__restrict__ w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) w[i] = btag[i] ? 0.0 : 1.0;
}

// *out = x[0] - sum_j lapP[j][0] p[idx[j][0]] (ELL [k][n]), one warp
__global__ void k_row0_residual(int n, int k, const int *__restrict__ idx, const double *__restrict__ lapP,
                                const double *__restrict__ x, const double *__restrict__ p, double *__restrict__ out)
{
    const int lane = threadIdx.x;
    double v = 0.0;
    for (int j = lane; j < k; j += 32) v += lapP[(long)j * n] * p[idx[(long)j * n]];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) *out = x[0] - v;
}

// p -= (rho0(b) / rho0(w)) p_w with s = {rho0(w), rho0(b)}
__global__ void k_compat_apply(int n, const double *__restrict__ s, const double *__restrict__ pw,
                               double *__restrict__ p)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] -= (s[1] / s[0]) * pw[i];
}

// D = p - p_hist when the history holds a previous pressure, else 0
__global__ void k_history_direction(int n, const double *__restrict__ p, const double *__restrict__ ph,
                                    const int *__restrict__ ok, double *__restrict__ d)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] = *ok ? p[i] - ph[i] : 0.0;
}

__global__ void k_set_flag(int *flag, int v) { *flag = v; }

// int16 offsets of a gather index from a per-row base node (base = nullptr: the row itself)
// ELL [k][ld] int16 offsets gidx - base (base: per-row node, or the row itself);
// padding rows (n <= i < ld) get offset 0
__global__ void k_make_offsets(int n, int ld, int k, const int *__restrict__ gidx, const int *__restrict__ base,
                               short *__restrict__ off, int *__restrict__ overflow)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)ld * k) return;
    const int i = (int)(t % ld);
    if (i >= n) { off[t] = 0; return; }
    const int d = gidx[t] - (base ? base[i] : i);
    if (d > 32767 || d < -32768) atomicOr(overflow, 1);
    off[t] = (short)d;
}

// The FP32 solver operator with each row's slots sorted by neighbour index
// (consecutive rows then gather from nearby addresses in the same slot), [k][ld]
// with ld >= n a multiple of 4; padding rows get weight 0 and index 0.
// The same sort gives the FP64 copy of the compact FP64 V-cycle (A64s, the
// level's slot order permuted the same way).
__global__ void __launch_bounds__(128) k_sort_slots(int n, int k, int ld, const int *__restrict__ idx,
                                                    const double *__restrict__ A64, int *__restrict__ sidx,
                                                    float *__restrict__ A32, double *__restrict__ A64s)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ld) return;
    if (i >= n) {
        for (int j = 0; j < k; j++) {
            sidx[(long)j * ld + i] = 0;
            A32[(long)j * ld + i] = 0.f;
            A64s[(long)j * ld + i] = 0.0;
        }
        return;
    }
    int c[kMaxK];
    short src[kMaxK];
    for (int j = 0; j < k; j++) {
        const int cj = idx[(long)j * n + i];
        int p = j;
        while (p > 0 && c[p - 1] > cj) { c[p] = c[p - 1]; src[p] = src[p - 1]; p--; }
        c[p] = cj;
        src[p] = (short)j;
    }
    for (int j = 0; j < k; j++) {
        const double a = A64[(long)src[j] * n + i];
        sidx[(long)j * ld + i] = c[j];
        A32[(long)j * ld + i] = (float)a;
        A64s[(long)j * ld + i] = a;
    }
}

// FP16 operator of the half-operator V-cycle (k_level_h4).  Interior row i's
// weights are scaled by 1 / A_ii (D^-1 A: unit diagonal, off-diagonal weights
// of order one) and rounded to FP16; the diagonal slot (offset 0) holds the
// row sum of the scaled weights instead, which k_level_h4 uses to apply the
// row in difference form.  One uint4 per stencil slot j and thread t (rows
// 128 g + 32 v + lane, g = t / 32, lane = t % 32, v = 0..3):
// {w_0, w_1 | w_2, w_3 | o_0, o_1 | o_2, o_3}, [k][ldi / 4];
// boundary and padding rows (which the level kernels do not use) get zero
// weights.  A value outside FP16's finite range sets *overflow.
__global__ void k_pack_half(int n, int k, int ld4, int ldi, const float *__restrict__ A32,
                            const short *__restrict__ off16, const float *__restrict__ dinv,
                            const uint8_t *__restrict__ btag, uint4 *__restrict__ W, int *__restrict__ overflow)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int q4 = ldi >> 2;
    if (t >= q4) return;
    const int ib = (t >> 5) * 128 + (t & 31);
    bool live[4];
    float di[4];
    double rs[4] = {0.0, 0.0, 0.0, 0.0};
    for (int v = 0; v < 4; v++) {
        const int i = ib + 32 * v;
        live[v] = i < n && !btag[i];
        di[v] = live[v] ? dinv[i] : 0.f;
    }
    for (int j = 0; j < k; j++)
        for (int v = 0; v < 4; v++)
            if (live[v]) rs[v] += (double)(A32[(long)j * ld4 + ib + 32 * v] * di[v]);
    for (int j = 0; j < k; j++) {
        unsigned h[4], o[4];
        for (int v = 0; v < 4; v++) {
            const int i = ib + 32 * v;
            float w = 0.f;
            o[v] = 0;
            if (i < n) {
                const long e = (long)j * ld4 + i;
                o[v] = (unsigned short)off16[e];
                if (live[v]) {
                    w = off16[e] == 0 ? (float)rs[v] : A32[e] * di[v];
                    if (!(fabsf(w) <= 65504.f)) atomicExch(overflow, 1);
                }
            }
            h[v] = __half_as_ushort(__float2half_rn(w));
        }
        W[(long)j * q4 + t] =
            make_uint4(h[0] | (h[1] << 16), h[2] | (h[3] << 16), o[0] | (o[1] << 16), o[2] | (o[3] << 16));
    }
}

// tile-major copy of an ELL array [k][ldin]: out[(t*k + j)*kTileRows + r] = in[j][t*kTileRows + r], zero past row n
template <class T>
__global__ void k_tile_major(int n, int k, int ld, int ldin, const T *__restrict__ in, T *__restrict__ out)
{
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long)k * ld) return;
    const int r = (int)(e % kTileRows);
    const long tj = e / kTileRows;
    const int j = (int)(tj % k);
    const long row = (tj / k) * kTileRows + r;
    out[e] = row < n ? in[(long)j * ldin + row] : T(0);
}

// decoded compact copy, row-major out: idx[i][j] = base_i + off[j][i] (base_i:
// the row itself, or base[i]) where off is given, else gidx[j][i]; w[i][j] = W[j][i]
__global__ void k_decode_compact(int n, int k, int ld, const short *__restrict__ off, const int *__restrict__ base,
                                 const int *__restrict__ gidx, const float *__restrict__ W, int *__restrict__ idx,
                                 float *__restrict__ w)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)n * k) return;
    const int i = (int)(t / k), j = (int)(t % k);
    const long e = (long)j * ld + i;
    idx[t] = off ? (base ? base[i] : i) + (int)off[e] : gidx[e];
    w[t] = W[e];
}

// compact copies of the boundary rows of the pinned operator: out[w][j] = A[j][list[w]]
__global__ void k_gather_rows(int nbl, const int *__restrict__ list, int n, int k, const int *__restrict__ idx,
                              const double *__restrict__ A, int *__restrict__ bidx, double *__restrict__ bA64,
                              float *__restrict__ bA32)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)nbl * k) return;
    const int w = (int)(t / k), j = (int)(t % k);
    const long o = (long)j * n + list[w];
    bidx[t] = idx[o];
    bA64[t] = A[o];
    bA32[t] = (float)A[o];
}

void knn_clouds(Level &L, int dim, cudaStream_t s)
{
    const int n = L.n, k = L.k, nb = L.nb;
    L.cloud.alloc((size_t)n * k);
    GridIndex gall, gint;
    grid_build(gall, n, L.x.p, L.y.p, L.z.p, nullptr, dim, s);
    if (n > nb)
        knn_query(gall, L.x.p, L.y.p, L.z.p, n - nb, L.x.p + nb, L.y.p + nb, L.z.p + nb, nullptr, k, 0,
                  L.cloud.p + (size_t)nb * k, k, s);
    if (nb > 0) {
        grid_build(gint, n, L.x.p, L.y.p, L.z.p, L.btag.p, dim, s);
        knn_query(gint, L.x.p, L.y.p, L.z.p, nb, L.x.p, L.y.p, L.z.p, nullptr, k, 1, L.cloud.p, k, s);
    }
    MGM_CUDA(cudaStreamSynchronize(s));
}

void nearest_of(const Level &T, const Level &S, int dim, DBuf<int> &out, cudaStream_t s)
{
    GridIndex g;
    grid_build(g, S.n, S.x.p, S.y.p, S.z.p, nullptr, dim, s);
    out.alloc(T.n);
    knn_query(g, S.x.p, S.y.p, S.z.p, T.n, T.x.p, T.y.p, T.z.p, nullptr, 1, 0, out.p, 1, s);
    MGM_CUDA(cudaStreamSynchronize(s));
}

// ELL transfer matrix from row-major weights (target rows [nt][ks]) with gather through src cloud
void build_transfer(const Level &T, const Level &S, const DBuf<int> &pts, int rows_from, int only_interior, int dim,
                    int phs, DBuf<int> &gidx, DBuf<double> &w64, DBuf<float> *w32, cudaStream_t s)
{
    const int nt = T.n, ks = S.k;
    DBuf<double> rm((size_t)nt * ks);
    Monomials mono = monomials(dim, S.poly);
    transfer_weights(nt, T.x.p, T.y.p, T.z.p, T.btag.p, pts.p, rows_from, only_interior, ks, dim, phs, mono, S.x.p,
                     S.y.p, S.z.p, S.cloud.p, rm.p, s);
    w64.alloc((size_t)nt * ks);
    transpose_rowmajor_to_ell_d(rm.p, w64.p, nt, ks, s);
    gidx.alloc((size_t)nt * ks);
    k_gather_idx<<<blocks_for((long)nt * ks, 256), 256, 0, s>>>(nt, ks, pts.p, S.cloud.p, gidx.p);
    MGM_LAUNCHED();
    if (w32) {
        w32->alloc((size_t)nt * ks);
        convert_d2f(w64.p, w32->p, (long)nt * ks, s);
    }
    MGM_CUDA(cudaStreamSynchronize(s));
}

template <class T>
std::vector<SolveLevel<T>> solve_levels(mgm_ctx *c);

template <>
std::vector<SolveLevel<double>> solve_levels<double>(mgm_ctx *c)
{
    std::vector<SolveLevel<double>> out;
    for (int l = 0; l < c->nl; l++) {
        Level &L = c->L[l];
        SolveLevel<double> S{};
        S.n = L.n; S.k = L.k; S.ld = L.n; S.nb_list = L.nbl;
        S.idx = L.idx.p; S.A = L.A64.p; S.dinv = L.dinv64.p; S.btag = L.btag.p; S.bnd_list = L.bnd_list.p;
        S.bnd_idx = L.bnd_idx.p; S.bnd_A = L.bnd_A64.p;
        S.r = L.r64.p; S.e = L.e64.p; S.e2 = L.e64b.p; S.d = L.d64.p; S.q = L.q64.p;
        S.kr = l > 0 ? c->L[l - 1].k : 0; S.r_idx = L.s_r_idx.p; S.r_w = L.s_r_w64.p;
        S.kp = l < c->nl - 1 ? c->L[l + 1].k : 0; S.p_idx = L.s_p_idx.p; S.p_w = L.s_p_w64.p;
        S.lmax = L.lmax;
        if (c->compact) {
            // the FP32 path's layout with FP64 weights: slots sorted by
            // neighbour, int16 offsets, four rows per thread on large levels
            if (L.off_ok) { S.ld = L.ld4; S.idx = L.sidx.p; S.A = L.A64s.p; S.off = L.off16.p; }
            S.r_off = L.r_off_ok ? L.r_off16.p : nullptr; S.r_base = L.rpts.p;
            S.p_off = L.p_off_ok ? L.p_off16.p : nullptr; S.p_base = L.ppts.p;
        }
        out.push_back(S);
    }
    return out;
}

template <>
std::vector<SolveLevel<float>> solve_levels<float>(mgm_ctx *c)
{
    std::vector<SolveLevel<float>> out;
    for (int l = 0; l < c->nl; l++) {
        Level &L = c->L[l];
        SolveLevel<float> S{};
        S.n = L.n; S.k = L.k; S.ld = L.ld4; S.nb_list = L.nbl;
        S.idx = L.sidx.p; S.A = L.A32.p; S.dinv = L.dinv32.p; S.btag = L.btag.p; S.bnd_list = L.bnd_list.p;
        S.bnd_idx = L.bnd_idx.p; S.bnd_A = L.bnd_A32.p;
        S.r = L.r32.p; S.e = L.e32.p; S.e2 = L.e32b.p; S.d = L.d32.p; S.q = L.q32.p;
        S.kr = l > 0 ? c->L[l - 1].k : 0; S.r_idx = L.s_r_idx.p; S.r_w = L.s_r_w32.p;
        S.kp = l < c->nl - 1 ? c->L[l + 1].k : 0; S.p_idx = L.s_p_idx.p; S.p_w = L.s_p_w32.p;
        S.lmax = L.lmax;
        if (c->compact) {
            S.off = L.off_ok ? L.off16.p : nullptr;
            S.r_off = L.r_off_ok ? L.r_off16.p : nullptr; S.r_base = L.rpts.p;
            S.p_off = L.p_off_ok ? L.p_off16.p : nullptr; S.p_base = L.ppts.p;
            if (c->use_tma && L.ldt > 0) {
                S.At = L.A32t.p; S.offt = L.off16t.p; S.ldt = L.ldt; S.tma_err = c->tma_err.p;
            }
            if (c->half_operator && L.h_ok) { S.W16 = L.W16.p; S.ldi = L.ldi; }
        }
        out.push_back(S);
    }
    return out;
}

StepArgs step_args(mgm_ctx *c)
{
    Level &L = c->L[0];
    StepArgs a{};
    a.n = L.n; a.k = L.k; a.idx = L.idx.p;
    a.Dx = L.Dx.p; a.Dy = L.Dy.p; a.Dz = L.Dz.p; a.lap = L.lap.p;
    a.btag = L.btag.p; a.nx = L.nx.p; a.ny = L.ny.p; a.nz = L.nz.p;
    a.u = c->u.p; a.v = c->v.p; a.w = c->w.p; a.u_new = c->u_new.p; a.v_new = c->v_new.p; a.w_new = c->w_new.p;
    a.p = L.p.p; a.source = L.src.p; a.dpdn = c->dpdn.p;
    a.dt = c->dt; a.nu = c->nu; a.rho = c->rho;
    return a;
}

std::vector<RefLevel> ref_levels(mgm_ctx *c)
{
    std::vector<RefLevel> out;
    for (int l = 0; l < c->nl; l++) {
        Level &L = c->L[l];
        RefLevel R{};
        R.n = L.n; R.k = L.k; R.idx = L.idx.p; R.lap = L.lap.p; R.lapP = L.lapP.p; R.btag = L.btag.p;
        R.p = L.p.p; R.ptmp = L.ptmp.p; R.src = L.src.p; R.res = L.res.p;
        R.r_idx = L.ref_r_idx.p; R.restr = L.ref_restr.p; R.p_idx = L.ref_p_idx.p; R.prol = L.ref_prol.p;
        out.push_back(R);
    }
    return out;
}

}  // namespace

// learned warm start (mpnn.cu)
namespace mgm {
bool warm_start_enabled(mgm_ctx *c);
template <class T>
void warm_direction(mgm_ctx *c, const double *b, const double *p, const double *dp, T *out, cudaStream_t s);
void destroy_mpnn(mgm_ctx *c);
}  // namespace mgm

namespace {

void drop_step_graphs(mgm_ctx *c);

// Whether a cooperative kernel may sit in a conditional node's body graph
// (the step graph puts the fused coarse V-cycle there): one is captured into
// a WHILE body (condition 0) and the graph instantiated, never launched.
bool cooperative_in_conditional_ok(mgm_ctx *c)
{
    cudaStream_t s = c->s, bs = c->s_body[0];
    bool ok = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        return false;
    }
    cudaGraph_t g = nullptr, body = nullptr;
    cudaStreamCaptureStatus cst;
    unsigned long long id = 0;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaGraphConditionalHandle h;
    ok = cudaStreamGetCaptureInfo(s, &cst, &id, &g, &deps, &ndeps) == cudaSuccess && g &&
         cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        ok = cudaGraphAddNode(&node, g, deps, ndeps, &np) == cudaSuccess &&
             cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies) == cudaSuccess;
        if (ok) body = np.conditional.phGraph_out[0];
    }
    if (ok && cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
                  cudaSuccess) {
        const bool launched = launch_coop_probe(bs) == cudaSuccess;
        cudaGraph_t out = nullptr;
        ok = cudaStreamEndCapture(bs, &out) == cudaSuccess && launched;
    } else {
        ok = false;
    }
    cudaGraph_t whole = nullptr;
    const bool ended = cudaStreamEndCapture(s, &whole) == cudaSuccess;
    cudaGraphExec_t x = nullptr;
    ok = ok && ended && whole && cudaGraphInstantiate(&x, whole, 0) == cudaSuccess;
    if (x) cudaGraphExecDestroy(x);
    if (whole) cudaGraphDestroy(whole);
    cudaGetLastError();  // a refused capture leaves no sticky error; clear the last one
    return ok;
}

FusedCtl fused_ctl(mgm_ctx *c)
{
    FusedCtl f;
    f.on = c->fused_coarse && c->fused_blocks > 0;
    f.blocks = c->fused_blocks;
    f.bar = c->fused_bar.p;
    f.err = c->tma_err.p;
    return f;
}

// a level kernel's bounded wait ran out (tile-streamed copies, the fused
// coarse V-cycle's grid barrier): clear the flags and report
void check_wait_flags(mgm_ctx *c, cudaStream_t s)
{
    if (!c->tma_err.p) return;
    int h_err = 0;
    c->tma_err.download(&h_err, 1, s);
    MGM_CUDA(cudaStreamSynchronize(s));
    if (h_err) {
        c->tma_err.zero(s);
        c->fused_bar.zero(s);
        MGM_CUDA(cudaStreamSynchronize(s));
        throw Error{MGM_ERR_TIMEOUT, "Poisson solve: a level kernel's bounded wait ran out (tile copies or the "
                                     "fused coarse V-cycle's grid barrier)"};
    }
}

void drop_graphs(mgm_ctx *c)
{
    drop_step_graphs(c);
    for (auto &g : c->vg) {
        if (g.x) cudaGraphExecDestroy(g.x);
        if (g.g) cudaGraphDestroy(g.g);
        g = mgm_ctx::VGraph();
    }
}

// One V-cycle: replayed from a captured CUDA graph (about a hundred kernels,
// most of them on launch-latency-bound coarse levels).  Returns the level-0
// correction buffer.
template <class T>
const T *run_vcycle(mgm_ctx *c, std::vector<SolveLevel<T>> &levels, const CoarseSolve<T> &cs)
{
    cudaStream_t s = c->s;
    if (!c->use_graphs) {
        const FusedCtl fc = fused_ctl(c);
        vcycle<T>(levels, cs, c->cheb_deg, c->cheb_ratio, s, &c->prof, c->chain_launches, &fc);
        return levels[0].e;
    }
    auto &G = c->vg[sizeof(T) == 4 ? 1 : 0];
    if (G.x && G.prof != c->prof.on) {
        cudaGraphExecDestroy(G.x);
        cudaGraphDestroy(G.g);
        G = mgm_ctx::VGraph();
    }
    if (!G.x) {
        std::vector<SolveLevel<T>> cap = levels;
        if (c->prof.on) {
            MGM_CUDA(cudaStreamSynchronize(s));
            c->prof.harvest();
        }
        const size_t first = c->prof.used;
        const long long launches_before = g_launches;
        MGM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        try {
            const FusedCtl fc = fused_ctl(c);
            vcycle<T>(cap, cs, c->cheb_deg, c->cheb_ratio, s, c->prof.on ? &c->prof : nullptr, c->chain_launches, &fc);
        } catch (...) {
            cudaGraph_t junk = nullptr;
            cudaStreamEndCapture(s, &junk);
            if (junk) cudaGraphDestroy(junk);
            throw;
        }
        MGM_CUDA(cudaStreamEndCapture(s, &G.g));
        MGM_CUDA(cudaGraphInstantiate(&G.x, G.g, 0));
        // captured launches did not run: count them once per replay instead
        G.kernels = g_launches - launches_before;
        g_launches = launches_before;
        G.out = (void *)cap[0].e;
        G.prof = c->prof.on;
        G.ev_first = first;
        G.ev_pairs = (c->prof.used - first) / 2;
        // the graph owns these event slots from now on
        c->prof.used = first;
        if (G.prof) {
            // keep the slots out of the eager recorder's way
            c->prof.used = first + 2 * G.ev_pairs;
        }
    }
    MGM_CUDA(cudaGraphLaunch(G.x, s));
    g_launches += G.kernels;
    return (const T *)G.out;
}

// ---------------------------------------------------------------------------
// Flexible GMRES(m) in FP64 right-preconditioned by one V-cycle in precision
// T.  Solves A p = b (pinned level-0 operator); p is the initial guess.
//
// Every scalar of the iteration lives on the device (FgState) and is updated
// by small kernels, so the same kernel sequence runs in two forms:
//  * host loops: after each restart cycle's start and each Arnoldi step the
//    host reads the loop flags (go_outer, go_inner) of the state's head;
//  * captured: the two loops become WHILE conditional nodes whose conditions
//    the same kernels set on the device (cudaGraphSetConditional), so the
//    whole solve (and the whole fractional step around it) is one graph
//    with no host round trip.
// Both forms launch the same kernels in the same order and give the same bits.
// ---------------------------------------------------------------------------
constexpr int kMaxRestarts = 4;

template <class T>
struct FgRun {
    mgm_ctx *c;
    std::vector<SolveLevel<T>> levels;
    CoarseSolve<T> cs;
    T *Z;
    double *V;
    long ld;
    int n, k, nbres;
    FgState *st;
    const double *b;
    double *p;
};

// the flags of the state's head, read by the host loops
const FgState &read_fg_head(mgm_ctx *c)
{
    MGM_CUDA(cudaMemcpyAsync(c->h_fg, c->fg.p, kFgHead, cudaMemcpyDeviceToHost, c->s));
    MGM_CUDA(cudaStreamSynchronize(c->s));
    return *c->h_fg;
}

// Adds a WHILE conditional node at the current capture position of stream s
// and returns its body graph.  create: a new handle *h on the graph s
// captures into, its condition reset to `dflt` at every launch of the graph;
// else *h is an existing handle of that graph.
cudaGraph_t add_while_node(cudaStream_t s, bool create, unsigned dflt, cudaGraphConditionalHandle *h)
{
    cudaStreamCaptureStatus cst;
    unsigned long long id = 0;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    MGM_CUDA(cudaStreamGetCaptureInfo(s, &cst, &id, &g, &deps, &ndeps));
    MGM_REQUIRE(cst == cudaStreamCaptureStatusActive && g, "add_while_node: stream is not capturing");
    if (create) MGM_CUDA(cudaGraphConditionalHandleCreate(h, g, dflt, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = *h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    MGM_CUDA(cudaGraphAddNode(&node, g, deps, ndeps, &np));
    MGM_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    return np.conditional.phGraph_out[0];
}

// captures body(bs) into a conditional node's body graph on side stream bs
template <class F>
void capture_body(cudaGraph_t body, cudaStream_t bs, F &&fn)
{
    MGM_CUDA(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    try {
        fn();
    } catch (...) {
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(bs, &junk);
        throw;
    }
    cudaGraph_t out = nullptr;
    MGM_CUDA(cudaStreamEndCapture(bs, &out));
}

// one Arnoldi step: z_j = M v_j (V-cycle), w = A z_j, classical Gram-Schmidt
// (projections and |w|^2 in one pass, the update with the norm of the result
// in a second, a re-orthogonalisation pass only when the first cancelled more
// than 1 - 1/sqrt(2) of |w|: the Daniel-Gragg-Kaufman-Stewart test), the
// Givens update and the convergence test
template <class T>
void arnoldi_step(FgRun<T> &R, cudaStream_t s, FgHandles hd, bool captured)
{
    mgm_ctx *c = R.c;
    Level &L0 = c->L[0];
    fg_load<T>(R.n, R.V, R.ld, R.st, R.levels[0].r, s);
    const T *z;
    if (captured) {
        const FusedCtl fc = fused_ctl(c);
        vcycle<T>(R.levels, R.cs, c->cheb_deg, c->cheb_ratio, s, nullptr, c->chain_launches, &fc);
        z = R.levels[0].e;
    } else {
        z = run_vcycle<T>(c, R.levels, R.cs);
    }
    fg_store<T>(R.n, z, R.Z, R.ld, R.st, s);
    fg_apply<T>(R.n, R.k, L0.idx.p, L0.A64.p, R.Z, R.ld, R.st, R.V, s);
    fg_gram_schmidt(R.n, R.V, R.ld, R.st, 0, c->kpart.p, s);
    fg_dgks(R.st, s);
    fg_gram_schmidt(R.n, R.V, R.ld, R.st, 1, c->kpart.p, s);
    fg_scale_w(R.n, R.V, R.ld, R.st, s);
    fg_arnoldi_end(R.st, hd, s);
    if (!captured && c->prof.on) {
        // the events of this V-cycle must have completed before they are read
        MGM_CUDA(cudaStreamSynchronize(c->s));
        auto &G = c->vg[sizeof(T) == 4 ? 1 : 0];
        if (c->use_graphs && G.x && G.prof) c->prof.harvest_graph(G.ev_first, G.ev_pairs);
        else c->prof.harvest();
    }
}

// one restart cycle: r = b - A p into V_0, the cycle's start (norms,
// convergence test, g = beta e_0), the Arnoldi steps, y = H^-1 g, p += Z y
template <class T>
void restart_cycle(FgRun<T> &R, cudaStream_t s, FgHandles hd, bool captured, long long *k_inner)
{
    mgm_ctx *c = R.c;
    Level &L0 = c->L[0];
    resid64(R.n, R.k, L0.idx.p, L0.A64.p, R.b, R.p, R.V, c->kpart.p, s);
    fg_begin(R.st, c->kpart.p, R.nbres, hd, s);
    fg_scale0(R.n, R.V, R.st, s);
    if (captured) {
        // the inner handle exists already: fg_begin above sets it
        cudaGraph_t body = add_while_node(s, false, 0, &hd.inner);
        cudaStream_t bs = c->s_body[1];
        const long long before = g_launches;
        capture_body(body, bs, [&] { arnoldi_step<T>(R, bs, hd, true); });
        if (k_inner) *k_inner = g_launches - before;
        g_launches = before;
    } else {
        while (read_fg_head(c).go_inner) arnoldi_step<T>(R, s, hd, false);
    }
    fg_solve_y(R.st, hd, s);
    fg_combine<T>(R.n, R.Z, R.ld, R.st, R.p, s);
}

// The initial guess of a step's solve (mgm_set_initial_guess).  Directions,
// staged in the Krylov basis: D0 = p - p_hist, the last pressure increment
// (zero when there is no history), and with the learned guess D1 = the
// network's predicted increment.  The network's output carries BF16-level
// grid-scale noise that the Laplacian amplifies, so D1 is first cleaned by
// Chebyshev smoothing of A e = b - A (p + D1) on the fine level (D1 += e).
// Then p += D c with c minimising |b - A (p + D c)|_2 (normal equations of
// the 1 or 2 columns A D; a zero or collinear column is dropped), which is
// never worse than p itself; the FGMRES then runs unchanged to the
// tolerance.  Every scalar stays on the device.
template <class T>
void initial_guess(FgRun<T> &R, bool learned, cudaStream_t s)
{
    mgm_ctx *c = R.c;
    Level &L0 = c->L[0];
    const int n = R.n, k = R.k;
    const long ld = R.ld;
    double *r0 = R.V, *D0 = R.V + ld, *D1 = R.V + 2 * ld, *AD0 = R.V + 3 * ld, *AD1 = R.V + 4 * ld;
    double *ks = c->kscal.p;
    const int nd = learned ? 2 : 1;
    k_history_direction<<<blocks_for(n, 256), 256, 0, s>>>(n, R.p, c->p_hist.p, c->hist_ok.p, D0);
    MGM_LAUNCHED();
    if (learned) {
        warm_direction<double>(c, R.b, R.p, D0, D1, s);
        if (c->warm_smooth_steps > 0) {
            double *pd = AD0;
            copy_out<double>(n, R.p, pd, s);
            set_scalar(ks, 1.0, s);
            combine<double>(n, 1, D1, ld, ks, pd, s);                        // pd = p + D1
            resid64(n, k, L0.idx.p, L0.A64.p, R.b, pd, r0, c->kpart.p, s);    // r0 = b - A (p + D1)
            copy_convert<T>(n, r0, R.levels[0].r, s);
            const T *e = smooth_from_zero<T>(R.levels[0], c->warm_smooth_steps, c->cheb_ratio, s, c->chain_launches);
            combine<T>(n, 1, e, ld, ks, D1, s);                              // D1 += e
        }
    }
    resid64(n, k, L0.idx.p, L0.A64.p, R.b, R.p, r0, c->kpart.p, s);
    apply64<double>(n, k, L0.idx.p, L0.A64.p, D0, AD0, s);
    if (learned) apply64<double>(n, k, L0.idx.p, L0.A64.p, D1, AD1, s);
    multidot(n, nd, AD0, ld, r0, c->kpart.p, ks, s);             // ks[i] = AD_i . r0
    multidot(n, nd, AD0, ld, AD0, c->kpart.p, ks + 2, s);        // ks[2 + i] = AD_i . AD0
    if (learned) multidot(n, nd, AD0, ld, AD1, c->kpart.p, ks + 4, s);  // ks[4 + i] = AD_i . AD1
    fg_guess_coefficients(R.st, ks, nd, s);                      // ks[6 .. 6 + nd)
    combine<double>(n, nd, D0, ld, ks + 6, R.p, s);
}

// Enqueues the solve on c->s.  captured: c->s is capturing a graph and the
// loops become conditional nodes (kernel counts of the loop bodies into
// k_outer / k_inner); else host loops, and the result is checked here.
// guesses: the step's initial guess (mgm_set_initial_guess) is applied first.
template <class T>
void fgmres(mgm_ctx *c, const double *b, double *p, bool captured = false, long long *k_outer = nullptr,
            long long *k_inner = nullptr, bool guesses = false)
{
    cudaStream_t s = c->s;
    Level &L0 = c->L[0];
    FgRun<T> R;
    R.c = c;
    R.n = L0.n;
    R.k = L0.k;
    R.ld = L0.n;
    R.nbres = blocks_for(L0.n, 256);
    R.levels = solve_levels<T>(c);
    R.cs.n = c->L[c->nl - 1].n;
    if constexpr (sizeof(T) == 8) R.cs.inv = (const T *)c->cinv64.p; else R.cs.inv = (const T *)c->cinv32.p;
    R.Z = sizeof(T) == 8 ? (T *)c->Z64.p : (T *)c->Z32.p;
    R.V = c->V.p;
    R.st = c->fg.p;
    R.b = b;
    R.p = p;
    const int m = std::min(c->max_iters, kMaxKrylov);
    fg_init(R.st, m, c->max_iters * (kMaxRestarts + 1), kMaxRestarts, c->tol, s);
    if (guesses) {
        MGM_REQUIRE(m >= 4, "initial guesses need max_iters >= 4 (their directions are staged in the Krylov basis)");
        initial_guess<T>(R, warm_start_enabled(c), s);
    }
    FgHandles hd;
    if (captured) {
        hd.use = 1;
        cudaGraph_t body = add_while_node(s, true, 1, &hd.outer);
        // the inner node lives in the outer body: its handle belongs to that graph
        MGM_CUDA(cudaGraphConditionalHandleCreate(&hd.inner, body, 0, 0));
        cudaStream_t bs = c->s_body[0];
        const long long before = g_launches;
        long long kin = 0;
        capture_body(body, bs, [&] { restart_cycle<T>(R, bs, hd, true, &kin); });
        if (k_outer) *k_outer = g_launches - before;
        if (k_inner) *k_inner = kin;
        g_launches = before;
        fg_final(R.st, s);
        return;
    }
    do {
        restart_cycle<T>(R, s, hd, false, nullptr);
    } while (read_fg_head(c).go_outer);
    fg_final(R.st, s);
    const FgState &h = read_fg_head(c);
    check_wait_flags(c, s);
    c->last_iters = h.vcycles;  // V-cycles (learned directions are not V-cycles)
    c->last_relres = h.relres;
    c->last_learned_alpha = h.alpha;
    if (h.status == FG_NONFINITE) throw Error{MGM_ERR_DIVERGED, "Poisson solve: non-finite residual"};
    if (h.status == FG_NOT_CONVERGED)
        throw Error{MGM_ERR_DIVERGED, "Poisson solve did not reach the tolerance (rel. residual " +
                                          std::to_string(h.relres) + " after " + std::to_string(h.total_it) +
                                          " V-cycles)"};
}

// p_w and rho0(w) of the compatible right-hand sides, after every set-up
void ensure_compat(mgm_ctx *c)
{
    if (c->compat_ready) return;
    Level &L0 = c->L[0];
    const int n = L0.n;
    cudaStream_t s = c->s;
    c->compat_pw.alloc(n);
    c->compat_s.alloc(2);
    DBuf<double> w(n);
    k_interior_indicator<<<blocks_for(n, 256), 256, 0, s>>>(n, L0.btag.p, w.p);
    MGM_LAUNCHED();
    copy_out<double>(n, w.p, c->bvec.p, s);
    k_zero_pinned<<<1, 1, 0, s>>>(c->bvec.p);
    MGM_LAUNCHED();
    c->compat_pw.zero(s);
    // p_w carries the pin's singular response to an incompatible source, so
    // its FP64 residual floors near the solver tolerance on fine levels; it
    // enters every solution scaled by alpha (the source's incompatible
    // fraction, ~1e-4 of |b|), so a relative residual of 1e-6 adds ~1e-10 |b|
    const double tol = c->tol;
    c->tol = std::max(tol, 1e-6);
    c->warm_suspended = true;
    try {
        fgmres<double>(c, c->bvec.p, c->compat_pw.p);
    } catch (...) {
        c->tol = tol;
        c->warm_suspended = false;
        throw;
    }
    c->tol = tol;
    c->warm_suspended = false;
    k_row0_residual<<<1, 32, 0, s>>>(n, L0.k, L0.idx.p, L0.lapP.p, w.p, c->compat_pw.p, c->compat_s.p);
    MGM_LAUNCHED();
    double rw = 0.0;
    c->compat_s.download(&rw, 1, s);
    MGM_CUDA(cudaStreamSynchronize(s));
    MGM_REQUIRE(std::isfinite(rw) && rw != 0.0,
                "compatible right-hand sides: the row-0 residual of the interior indicator is zero or not finite");
    c->last_iters = 0;
    c->compat_ready = true;
}

// The Poisson solve of a step on L0.src -> L0.p.  captured: enqueued into a
// graph being captured on c->s (the loops as conditional nodes, kernel counts
// of the loop bodies into k_outer / k_inner).
// step: a fractional step's solve, which applies the initial guess of
// mgm_set_initial_guess and keeps the pressure history
void poisson(mgm_ctx *c, int mode, bool timple = false, bool captured = false, long long *k_outer = nullptr,
             long long *k_inner = nullptr, bool step = false)
{
    Level &L0 = c->L[0];
    if (mode == MGM_MODE_REFERENCE) {
        MGM_REQUIRE(c->have_ref_transfer || c->nl == 1, "reference mode needs mgm_setup(..., MGM_SETUP_REFERENCE_TRANSFER)");
        auto R = ref_levels(c);
        const double w1 = (double)c->omega, w2 = (double)(1 - c->omega);
        ref_multigrid(R, w1, w2, c->num_relax, c->num_vcycles, c->s, timple ? REF_TIMPLE : REF_FS);
        return;
    }
    if (mode != MGM_MODE_FP64 && mode != MGM_MODE_FP32_IR) throw Error{MGM_ERR_ARG, "unknown Poisson mode"};
    if (c->compat) MGM_REQUIRE(c->compat_ready || !captured, "poisson: compatible right-hand sides not prepared");
    if (c->compat) ensure_compat(c);
    // b = source with the pinned row's rhs 0 (boundary rows keep their (zero) source)
    copy_out<double>(L0.n, L0.src.p, c->bvec.p, c->s);
    k_zero_pinned<<<1, 1, 0, c->s>>>(c->bvec.p);
    MGM_LAUNCHED();
    const bool guesses = step && c->guess_flags != 0 && !c->warm_suspended;
    if (step) copy_out<double>(L0.n, L0.p.p, c->p_start.p, c->s);
    if (mode == MGM_MODE_FP64) fgmres<double>(c, c->bvec.p, L0.p.p, captured, k_outer, k_inner, guesses);
    else fgmres<float>(c, c->bvec.p, L0.p.p, captured, k_outer, k_inner, guesses);
    if (step) {
        // the pressure this solve started from is p_prev2 of the next step
        copy_out<double>(L0.n, c->p_start.p, c->p_hist.p, c->s);
        k_set_flag<<<1, 1, 0, c->s>>>(c->hist_ok.p, 1);
        MGM_LAUNCHED();
    }
    if (c->compat) {
        k_row0_residual<<<1, 32, 0, c->s>>>(L0.n, L0.k, L0.idx.p, L0.lapP.p, L0.src.p, L0.p.p, c->compat_s.p + 1);
        MGM_LAUNCHED();
        k_compat_apply<<<blocks_for(L0.n, 256), 256, 0, c->s>>>(L0.n, c->compat_s.p, c->compat_pw.p, L0.p.p);
        MGM_LAUNCHED();
    }
}

void ensure_events(mgm_ctx *c)
{
    for (auto &e : c->ev)
        if (!e) MGM_CUDA(cudaEventCreate(&e));
}

// The kernels of one fractional step (fractional_step_explicit) on c->s:
// momentum, divergence, the Poisson solve between two device time marks,
// the velocity correction and its steady-state error, and the error's copy
// into c->h_pinned[0].
void step_kernels(mgm_ctx *c, int mode, bool captured, long long *k_outer = nullptr, long long *k_inner = nullptr)
{
    StepArgs a = step_args(c);
    launch_momentum(a, c->dim, c->s);
    launch_divergence(a, c->dim, c->s);
    fg_time_mark(c->fg.p, 0, c->s);
    poisson(c, mode, false, captured, k_outer, k_inner, true);
    fg_time_mark(c->fg.p, 1, c->s);
    launch_correct(a, c->dim, c->partial.p, c->scal.p, c->s);
    MGM_CUDA(cudaMemcpyAsync(c->h_pinned, c->scal.p, sizeof(double), cudaMemcpyDeviceToHost, c->s));
}

void drop_step_graphs(mgm_ctx *c)
{
    for (auto &g : c->sg) {
        if (g.x) cudaGraphExecDestroy(g.x);
        if (g.g) cudaGraphDestroy(g.g);
        g = mgm_ctx::StepGraph();
    }
}

bool step_graph_usable(mgm_ctx *c, int mode)
{
    return c->use_graphs && c->step_graphs && !c->prof.on && (mode == MGM_MODE_FP64 || mode == MGM_MODE_FP32_IR);
}

// The step graph of `mode`, captured on first use and whenever the settings
// it bakes in (dt through the kernels' arguments, the learned warm start,
// compatible right-hand sides) changed; solver settings drop it (drop_graphs).
mgm_ctx::StepGraph &step_graph(mgm_ctx *c, int mode)
{
    auto &G = c->sg[mode == MGM_MODE_FP32_IR ? 1 : 0];
    const int guess = c->guess_flags | (warm_start_enabled(c) ? 0x100 : 0);
    if (G.x && (G.guess != guess || G.compat != c->compat || G.dt != c->dt)) {
        cudaGraphExecDestroy(G.x);
        cudaGraphDestroy(G.g);
        G = mgm_ctx::StepGraph();
    }
    if (G.x) return G;
    if (c->compat) ensure_compat(c);
    MGM_CUDA(cudaStreamSynchronize(c->s));
    const long long before = g_launches;
    long long ko = 0, ki = 0;
    MGM_CUDA(cudaStreamBeginCapture(c->s, cudaStreamCaptureModeThreadLocal));
    try {
        step_kernels(c, mode, true, &ko, &ki);
    } catch (...) {
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(c->s, &junk);
        if (junk) cudaGraphDestroy(junk);
        g_launches = before;
        throw;
    }
    MGM_CUDA(cudaStreamEndCapture(c->s, &G.g));
    MGM_CUDA(cudaGraphInstantiate(&G.x, G.g, 0));
    G.k_top = g_launches - before;
    G.k_outer = ko;
    G.k_inner = ki;
    g_launches = before;
    G.guess = guess;
    G.compat = c->compat;
    G.dt = c->dt;
    return G;
}

// Launches nsteps fractional steps: replays of the step graph (no host
// synchronisation inside or between them) or, in reference mode, with
// profiling or with step graphs off, the host-driven step.  Returns the
// steady-state error of the last step; the Poisson time and V-cycles of the
// steps accumulate on the device (c->fg totals, cleared by the caller).
double run_steps_device(mgm_ctx *c, int mode, int nsteps)
{
    if (step_graph_usable(c, mode)) {
        auto &G = step_graph(c, mode);
        for (int t = 0; t < nsteps; t++) MGM_CUDA(cudaGraphLaunch(G.x, c->s));
        MGM_CUDA(cudaStreamSynchronize(c->s));
        const FgState &h = read_fg_head(c);
        g_launches += (long long)nsteps * G.k_top + h.cycles_total * G.k_outer + h.vcycles_total * G.k_inner;
        check_wait_flags(c, c->s);
        if (h.err_any & 1) throw Error{MGM_ERR_DIVERGED, "Poisson solve: non-finite residual"};
        if (h.err_any & 2) throw Error{MGM_ERR_DIVERGED, "Poisson solve did not reach the tolerance"};
        c->last_iters = h.vcycles;
        c->last_relres = h.relres;
        c->last_learned_alpha = h.alpha;
        return c->h_pinned[0];
    }
    for (int t = 0; t < nsteps; t++) {
        step_kernels(c, mode, false);
        MGM_CUDA(cudaStreamSynchronize(c->s));
        if (mode == MGM_MODE_REFERENCE) c->ref_vcycles_acc += c->num_vcycles;
    }
    return c->h_pinned[0];
}

// p_w of the compatible right-hand sides before a run of steps (so that its
// own solve is not counted in the steps' V-cycles)
void prepare_steps(mgm_ctx *c, int mode)
{
    if (c->compat && (mode == MGM_MODE_FP64 || mode == MGM_MODE_FP32_IR)) ensure_compat(c);
}

// one fractional step; Poisson time and V-cycles added to the context's counters
double step_timed(mgm_ctx *c, int mode)
{
    prepare_steps(c, mode);
    fg_clear_totals(c->fg.p, c->s);
    c->ref_vcycles_acc = 0;
    const double e = run_steps_device(c, mode, 1);
    const FgState &h = read_fg_head(c);
    c->poisson_ms_acc += h.t_ns * 1e-6;
    c->vcycles_acc += mode == MGM_MODE_REFERENCE ? c->ref_vcycles_acc : h.vcycles_total;
    return e;
}

void alloc_solver_buffers(mgm_ctx *c)
{
    const int n = c->L[0].n;
    const int m = std::min(c->max_iters, kMaxKrylov);
    c->V.alloc((size_t)(m + 1) * n);
    c->Z64.alloc((size_t)m * n);
    c->Z32.alloc((size_t)m * n);
    c->wv.alloc(n);
    c->wdir.alloc(n);
    if (c->p_start.n != (size_t)n) {
        c->p_start.alloc(n);
        c->p_hist.alloc(n);
        c->p_hist.zero(c->s);
    }
    if (!c->hist_ok.p) {
        c->hist_ok.alloc(1);
        c->hist_ok.zero(c->s);
    }
    c->bvec.alloc(n);
    c->kpart.alloc((size_t)std::max(2 * blocks_for(n, 256), (kMaxKrylov + 1) * dot_blocks(n)) + 16);
    c->kscal.alloc(3 * kMaxKrylov + 16);
    if (!c->fg.p) {
        c->fg.alloc(1);
        c->fg.zero(c->s);
    }
    if (!c->h_fg) MGM_CUDA(cudaMallocHost(&c->h_fg, sizeof(FgState)));
    if (!c->h_pinned) MGM_CUDA(cudaMallocHost(&c->h_pinned, sizeof(double) * (3 * kMaxKrylov + 16 + 2 * 65536)));
}

}  // namespace

namespace mgm {
// The Poisson solve of a step on L0.src -> L0.p (the TIMPLE step uses it for p').
void poisson_solve(mgm_ctx *c, int mode, bool timple) { poisson(c, mode, timple); }
// num_cycles reference-semantics V-cycles of one program's variant on every
// level's p, src and res (the heat-conduction program drives its own cycle)
void ref_cycles(mgm_ctx *c, RefVariant v, int num_cycles)
{
    MGM_REQUIRE(c->have_ref_transfer || c->nl == 1, "reference mode needs mgm_setup(..., MGM_SETUP_REFERENCE_TRANSFER)");
    auto R = ref_levels(c);
    const double w1 = (double)c->omega, w2 = (double)(1 - c->omega);
    ref_multigrid(R, w1, w2, c->num_relax, num_cycles, c->s, v);
}
}  // namespace mgm

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char *mgm_last_error(void) { return t_err.c_str(); }
int mgm_set_device(int device)
{
    return guard([&] { MGM_CUDA(cudaSetDevice(device)); });
}
long long mgm_kernel_launches(void) { return g_launches; }
int mgm_version(void) { return 1; }

int mgm_knn_cloud(int n, int nb, int dim, const double *x, const double *y, const double *z, const unsigned char *btag,
                  int k, int *cloud)
{
    return guard([&] {
        MGM_REQUIRE(n > 0 && nb >= 0 && nb <= n && k >= 1 && k <= kMaxK && (dim == 2 || dim == 3), "mgm_knn_cloud: bad sizes");
        MGM_REQUIRE(x && y && z && btag && cloud, "mgm_knn_cloud: null pointer");
        int ninterior = 0;
        for (int i = 0; i < n; i++) ninterior += btag[i] ? 0 : 1;
        MGM_REQUIRE(n >= k && (nb == 0 || ninterior >= k - 1), "mgm_knn_cloud: fewer candidate nodes than the stencil size");
        cudaStream_t s = tmp_stream();
        Level L;
        L.n = n; L.nb = nb; L.k = k;
        L.x.upload(x, n, s); L.y.upload(y, n, s); L.z.upload(z, n, s);
        L.btag.upload(btag, n, s);
        knn_clouds(L, dim, s);
        L.cloud.download(cloud, (size_t)n * k, s);
        MGM_CUDA(cudaStreamSynchronize(s));
    });
}

int mgm_nearest_points(int n1, const double *x1, const double *y1, const double *z1, int n2, const double *x2,
                       const double *y2, const double *z2, int dim, int *nearest)
{
    return guard([&] {
        MGM_REQUIRE(n1 >= 0 && n2 > 0, "mgm_nearest_points: bad sizes");
        if (n1 == 0) return;
        cudaStream_t s = tmp_stream();
        Level A, B;
        A.n = n1; B.n = n2;
        A.x.upload(x1, n1, s); A.y.upload(y1, n1, s); A.z.upload(z1, n1, s);
        B.x.upload(x2, n2, s); B.y.upload(y2, n2, s); B.z.upload(z2, n2, s);
        DBuf<int> out;
        nearest_of(A, B, dim, out, s);
        out.download(nearest, n1, s);
        MGM_CUDA(cudaStreamSynchronize(s));
    });
}

int mgm_bfs_order(int n, int k, const int *cloud, int *queue1)
{
    return guard([&] {
        MGM_REQUIRE(n > 0 && k >= 2, "mgm_bfs_order: bad sizes");
        for (long t = 0; t < (long)n * k; t++) MGM_REQUIRE(cloud[t] >= 0 && cloud[t] < n, "mgm_bfs_order: cloud index out of range");
        cudaStream_t s = tmp_stream();
        DBuf<int> dc, dq(n);
        dc.upload(cloud, (size_t)n * k, s);
        int reached = bfs_order(n, k, dc.p, dq.p, s);
        dq.download(queue1, n, s);
        MGM_CUDA(cudaStreamSynchronize(s));
        MGM_REQUIRE(reached == n, "mgm_bfs_order: stencil graph is disconnected (reached " + std::to_string(reached) +
                                      " of " + std::to_string(n) + " nodes)");
    });
}

int mgm_apply_order(int n, int k, const int *queue1, double *x, double *y, double *z, double *nx, double *ny, double *nz,
                    unsigned char *btag, int *cloud)
{
    return guard([&] {
        MGM_REQUIRE(n > 0 && k >= 1, "mgm_apply_order: bad sizes");
        cudaStream_t s = tmp_stream();
        DBuf<int> q, cl;
        DBuf<double> a[6];
        double *h[6] = {x, y, z, nx, ny, nz};
        DBuf<uint8_t> bt;
        q.upload(queue1, n, s);
        for (int t = 0; t < 6; t++) a[t].upload(h[t], n, s);
        bt.upload(btag, n, s);
        cl.upload(cloud, (size_t)n * k, s);
        apply_order(n, k, q.p, a[0].p, a[1].p, a[2].p, a[3].p, a[4].p, a[5].p, bt.p, cl.p, s);
        for (int t = 0; t < 6; t++) a[t].download(h[t], n, s);
        bt.download(btag, n, s);
        cl.download(cloud, (size_t)n * k, s);
        MGM_CUDA(cudaStreamSynchronize(s));
    });
}

int mgm_correct_normals(int n, int k, const double *x, const double *y, const double *z, const unsigned char *btag,
                        const int *cloud, double *nx, double *ny, double *nz)
{
    return guard([&] {
        cudaStream_t s = tmp_stream();
        DBuf<double> a[6];
        const double *in[3] = {x, y, z};
        double *io[3] = {nx, ny, nz};
        for (int t = 0; t < 3; t++) a[t].upload(in[t], n, s);
        for (int t = 0; t < 3; t++) a[3 + t].upload(io[t], n, s);
        DBuf<uint8_t> bt;
        DBuf<int> cl;
        bt.upload(btag, n, s);
        cl.upload(cloud, (size_t)n * k, s);
        correct_normals(n, k, a[0].p, a[1].p, a[2].p, bt.p, cl.p, a[3].p, a[4].p, a[5].p, s);
        for (int t = 0; t < 3; t++) a[3 + t].download(io[t], n, s);
        MGM_CUDA(cudaStreamSynchronize(s));
    });
}

int mgm_avg_dx(int n, int k, int dim, const double *x, const double *y, const double *z, const unsigned char *btag,
               const int *cloud, double *d_avg)
{
    return guard([&] {
        cudaStream_t s = tmp_stream();
        DBuf<double> a[3], out(1);
        const double *in[3] = {x, y, z};
        for (int t = 0; t < 3; t++) a[t].upload(in[t], n, s);
        DBuf<uint8_t> bt;
        DBuf<int> cl;
        bt.upload(btag, n, s);
        cl.upload(cloud, (size_t)n * k, s);
        avg_dx(n, k, dim, a[0].p, a[1].p, a[2].p, bt.p, cl.p, out.p, s);
        out.download(d_avg, 1, s);
        MGM_CUDA(cudaStreamSynchronize(s));
    });
}

int mgm_derivative_weights(int n, int k, int dim, int phs, int poly_degree, const double *x, const double *y,
                           const double *z, const double *nx, const double *ny, const double *nz,
                           const unsigned char *btag, const int *cloud, double *Dx, double *Dy, double *Dz, double *lap,
                           double *lapP)
{
    return guard([&] {
        MGM_REQUIRE(n > 0 && k >= 2 && (dim == 2 || dim == 3), "mgm_derivative_weights: bad sizes");
        MGM_REQUIRE(dim == 2 || Dz != nullptr, "mgm_derivative_weights: Dz required in 3D");
        for (long t = 0; t < (long)n * k; t++) MGM_REQUIRE(cloud[t] >= 0 && cloud[t] < n, "mgm_derivative_weights: cloud index out of range");
        cudaStream_t s = tmp_stream();
        Monomials mono = monomials(dim, poly_degree);
        DBuf<double> a[6];
        const double *in[6] = {x, y, z, nx, ny, nz};
        for (int t = 0; t < 6; t++) a[t].upload(in[t], n, s);
        DBuf<uint8_t> bt;
        DBuf<int> cl;
        bt.upload(btag, n, s);
        cl.upload(cloud, (size_t)n * k, s);
        DBuf<double> o[5];
        for (int t = 0; t < 5; t++) o[t].alloc((size_t)n * k);
        derivative_weights(n, k, dim, phs, mono, a[0].p, a[1].p, a[2].p, a[3].p, a[4].p, a[5].p, bt.p, cl.p, o[0].p,
                           o[1].p, dim == 3 ? o[2].p : nullptr, o[3].p, o[4].p, s);
        double *h[5] = {Dx, Dy, Dz, lap, lapP};
        for (int t = 0; t < 5; t++)
            if (h[t] && (t != 2 || dim == 3)) o[t].download(h[t], (size_t)n * k, s);
        MGM_CUDA(cudaStreamSynchronize(s));
    });
}

int mgm_transfer_weights(int nt, const double *tx, const double *ty, const double *tz, const unsigned char *tbtag,
                         const int *src_pt, int rows_from, int only_interior, int ns, int ks, int dim, int phs,
                         int poly_degree_src, const double *sx, const double *sy, const double *sz, const int *scloud,
                         double *W)
{
    return guard([&] {
        MGM_REQUIRE(nt >= 0 && ns > 0 && ks >= 2, "mgm_transfer_weights: bad sizes");
        for (int i = 0; i < nt; i++) MGM_REQUIRE(src_pt[i] >= 0 && src_pt[i] < ns, "mgm_transfer_weights: source point out of range");
        for (long t = 0; t < (long)ns * ks; t++) MGM_REQUIRE(scloud[t] >= 0 && scloud[t] < ns, "mgm_transfer_weights: cloud index out of range");
        if (nt == 0) return;
        cudaStream_t s = tmp_stream();
        Monomials mono = monomials(dim, poly_degree_src);
        DBuf<double> t3[3], s3[3], out((size_t)nt * ks);
        const double *ti[3] = {tx, ty, tz}, *si[3] = {sx, sy, sz};
        for (int q = 0; q < 3; q++) { t3[q].upload(ti[q], nt, s); s3[q].upload(si[q], ns, s); }
        DBuf<uint8_t> bt;
        DBuf<int> sp, cl;
        bt.upload(tbtag, nt, s);
        sp.upload(src_pt, nt, s);
        cl.upload(scloud, (size_t)ns * ks, s);
        transfer_weights(nt, t3[0].p, t3[1].p, t3[2].p, bt.p, sp.p, rows_from, only_interior, ks, dim, phs, mono,
                         s3[0].p, s3[1].p, s3[2].p, cl.p, out.p, s);
        out.download(W, (size_t)nt * ks, s);
        MGM_CUDA(cudaStreamSynchronize(s));
    });
}

int mgm_spmv(int n, int k, const double *D, const int *cloud, const double *f, double *out)
{
    return guard([&] {
        MGM_REQUIRE(n > 0 && k >= 1, "mgm_spmv: bad sizes");
        for (long t = 0; t < (long)n * k; t++) MGM_REQUIRE(cloud[t] >= 0 && cloud[t] < n, "mgm_spmv: cloud index out of range");
        cudaStream_t s = tmp_stream();
        DBuf<double> rm, W((size_t)n * k), fv, o(n);
        DBuf<int> cr, idx((size_t)n * k);
        rm.upload(D, (size_t)n * k, s);
        cr.upload(cloud, (size_t)n * k, s);
        fv.upload(f, n, s);
        transpose_rowmajor_to_ell_d(rm.p, W.p, n, k, s);
        transpose_rowmajor_to_ell_i(cr.p, idx.p, n, k, s);
        spmv_parity(n, k, W.p, idx.p, fv.p, o.p, s);
        o.download(out, n, s);
        MGM_CUDA(cudaStreamSynchronize(s));
    });
}

// ---------------------------------------------------------------------------
mgm_ctx *mgm_create(int dim, int phs_degree, int num_levels)
{
    mgm_ctx *c = nullptr;
    int st = guard([&] {
        MGM_REQUIRE(dim == 2 || dim == 3, "mgm_create: dim must be 2 or 3");
        MGM_REQUIRE(num_levels >= 1 && num_levels <= 16, "mgm_create: 1..16 levels");
        MGM_REQUIRE(phs_degree >= 1 && phs_degree <= 11, "mgm_create: phs degree out of range");
        int ndev = 0;
        MGM_CUDA(cudaGetDeviceCount(&ndev));
        MGM_REQUIRE(ndev > 0, "mgm_create: no CUDA device");
        std::unique_ptr<mgm_ctx> cc(new mgm_ctx());
        MGM_CUDA(cudaGetDevice(&cc->device));
        cc->dim = dim; cc->phs = phs_degree; cc->nl = num_levels;
        cc->L.resize(num_levels);
        MGM_CUDA(cudaStreamCreateWithFlags(&cc->s, cudaStreamNonBlocking));
        for (auto &bs : cc->s_body) MGM_CUDA(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking));
        c = cc.release();
    });
    return st == MGM_OK ? c : nullptr;
}

void mgm_destroy(mgm_ctx *c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->s) cudaStreamSynchronize(c->s);
    if (c->h_pinned) cudaFreeHost(c->h_pinned);
    if (c->h_fg) cudaFreeHost(c->h_fg);
    drop_graphs(c);
    destroy_mpnn(c);
    c->L.clear();
    for (auto &bs : c->s_body)
        if (bs) cudaStreamDestroy(bs);
    if (c->s) cudaStreamDestroy(c->s);
    delete c;
}

int mgm_set_level(mgm_ctx *c, int lev, int n, int nb, const double *x, const double *y, const double *z,
                  const double *nx, const double *ny, const double *nz, const unsigned char *btag, int poly_degree, int k)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(lev >= 0 && lev < c->nl, "mgm_set_level: level out of range");
        MGM_REQUIRE(n > 0 && nb >= 1 && nb <= n && k >= 2 && k <= kMaxK && poly_degree >= 0, "mgm_set_level: bad sizes");
        MGM_REQUIRE(x && y && z && nx && ny && nz && btag, "mgm_set_level: null pointer");
        for (int i = 0; i < n; i++)
            MGM_REQUIRE(std::isfinite(x[i]) && std::isfinite(y[i]) && std::isfinite(z[i]), "mgm_set_level: non-finite coordinate");
        int ninterior = 0;
        for (int i = 0; i < n; i++) ninterior += btag[i] ? 0 : 1;
        MGM_REQUIRE(ninterior >= k - 1 && n >= k, "mgm_set_level: fewer interior nodes than the stencil needs");
        Monomials mono = monomials(c->dim, poly_degree);
        MGM_REQUIRE(k + mono.np <= kMaxN, "mgm_set_level: k + num_poly_terms too large");
        Level &L = c->L[lev];
        L = Level();
        L.n = n; L.nb = nb; L.k = k; L.poly = poly_degree; L.np = mono.np;
        cudaStream_t s = c->s;
        L.x.upload(x, n, s); L.y.upload(y, n, s); L.z.upload(z, n, s);
        L.nx.upload(nx, n, s); L.ny.upload(ny, n, s); L.nz.upload(nz, n, s);
        L.btag.upload(btag, n, s);
        MGM_CUDA(cudaStreamSynchronize(s));
        c->setup_done = false;
    });
}

}  // extern "C"

namespace {

// read_complete_mesh_data (mesh_functions.h:914-928) after the reader: kNN
// clouds, breadth-first reorder, normals, average spacing, per level
void pipeline_geometry(mgm_ctx *c)
{
    cudaStream_t s = c->s;
    for (int l = 0; l < c->nl; l++) {
        Level &L = c->L[l];
        knn_clouds(L, c->dim, s);
        DBuf<int> q1(L.n);
        int reached = bfs_order(L.n, L.k, L.cloud.p, q1.p, s);
        MGM_REQUIRE(reached == L.n, "mgm_setup: stencil graph of level " + std::to_string(l) + " is disconnected");
        apply_order(L.n, L.k, q1.p, L.x.p, L.y.p, L.z.p, L.nx.p, L.ny.p, L.nz.p, L.btag.p, L.cloud.p, s);
        correct_normals(L.n, L.k, L.x.p, L.y.p, L.z.p, L.btag.p, L.cloud.p, L.nx.p, L.ny.p, L.nz.p, s);
        DBuf<double> d(1);
        avg_dx(L.n, L.k, c->dim, L.x.p, L.y.p, L.z.p, L.btag.p, L.cloud.p, d.p, s);
        d.download(&L.d_avg, 1, s);
        L.idx.alloc((size_t)L.n * L.k);
        transpose_rowmajor_to_ell_i(L.cloud.p, L.idx.p, L.n, L.k, s);
    }
    MGM_CUDA(cudaStreamSynchronize(s));
    // create_prolongation_and_restriction_matrices (mesh_functions.h:874-893): points
    for (int l = 0; l < c->nl; l++) {
        Level &L = c->L[l];
        nearest_of(L, l < c->nl - 1 ? c->L[l + 1] : L, c->dim, L.ppts, s);
        nearest_of(L, l > 0 ? c->L[l - 1] : L, c->dim, L.rpts, s);
    }
}

// transfer weights: the reference's rows (rows >= nb, optional) and the solver's rows
void pipeline_transfer(mgm_ctx *c, bool reference_rows)
{
    cudaStream_t s = c->s;
    for (int l = 0; l < c->nl; l++) {
        Level &L = c->L[l];
        if (l < c->nl - 1) {
            Level &C = c->L[l + 1];
            if (reference_rows)
                build_transfer(L, C, L.ppts, L.nb, 0, c->dim, c->phs, L.ref_p_idx, L.ref_prol, nullptr, s);
            build_transfer(L, C, L.ppts, 0, 0, c->dim, c->phs, L.s_p_idx, L.s_p_w64, &L.s_p_w32, s);
        }
        if (l > 0) {
            Level &F = c->L[l - 1];
            if (reference_rows)
                build_transfer(L, F, L.rpts, L.nb, 0, c->dim, c->phs, L.ref_r_idx, L.ref_restr, nullptr, s);
            build_transfer(L, F, L.rpts, 0, 1, c->dim, c->phs, L.s_r_idx, L.s_r_w64, &L.s_r_w32, s);
        }
    }
}

// create_derivative_matrices (rbf.h:401-421) on every level, into ELL
void pipeline_derivatives(mgm_ctx *c)
{
    cudaStream_t s = c->s;
    for (int l = 0; l < c->nl; l++) {
        Level &L = c->L[l];
        const size_t nk = (size_t)L.n * L.k;
        DBuf<double> rm[5];
        for (int t = 0; t < 5; t++) rm[t].alloc(nk);
        Monomials mono = monomials(c->dim, L.poly);
        derivative_weights(L.n, L.k, c->dim, c->phs, mono, L.x.p, L.y.p, L.z.p, L.nx.p, L.ny.p, L.nz.p, L.btag.p,
                           L.cloud.p, rm[0].p, rm[1].p, c->dim == 3 ? rm[2].p : nullptr, rm[3].p, rm[4].p, s);
        DBuf<double> *dst[5] = {&L.Dx, &L.Dy, &L.Dz, &L.lap, &L.lapP};
        for (int t = 0; t < 5; t++) {
            if (t == 2 && c->dim != 3) continue;
            dst[t]->alloc(nk);
            transpose_rowmajor_to_ell_d(rm[t].p, dst[t]->p, L.n, L.k, s);
        }
        MGM_CUDA(cudaStreamSynchronize(s));
    }
}

// pinned operators, boundary rows, smoother bounds, coarsest inverse, fields
void prepare_solver(mgm_ctx *c)
{
    cudaStream_t s = c->s;
    drop_graphs(c);
    c->compat_ready = false;
    for (int l = 0; l < c->nl; l++) {
        Level &L = c->L[l];
        const size_t nk = (size_t)L.n * L.k;
        L.ld4 = (L.n + 3) & ~3;
        const size_t nk4 = (size_t)L.ld4 * L.k;
        L.A64.alloc(nk); L.A32.alloc(nk4); L.A64s.alloc(nk4); L.sidx.alloc(nk4); L.dinv64.alloc(L.n);
        L.dinv32.alloc(L.n);
        k_pin_operator<<<blocks_for((long)nk, 256), 256, 0, s>>>(L.n, L.k, L.lapP.p, L.A64.p, L.dinv64.p,
                                                               L.dinv32.p);
        MGM_LAUNCHED();
        k_sort_slots<<<blocks_for(L.ld4, 128), 128, 0, s>>>(L.n, L.k, L.ld4, L.idx.p, L.A64.p, L.sidx.p, L.A32.p,
                                                            L.A64s.p);
        MGM_LAUNCHED();
        std::vector<uint8_t> hb(L.n);
        L.btag.download(hb.data(), L.n, s);
        MGM_CUDA(cudaStreamSynchronize(s));
        std::vector<int> bl;
        for (int i = 0; i < L.n; i++) if (hb[i]) bl.push_back(i);
        L.nbl = (int)bl.size();
        L.bnd_list.upload(bl.data(), bl.size(), s);
        L.bnd_idx.alloc((size_t)L.nbl * L.k);
        L.bnd_A64.alloc((size_t)L.nbl * L.k);
        L.bnd_A32.alloc((size_t)L.nbl * L.k);
        k_gather_rows<<<blocks_for((long)L.nbl * L.k, 256), 256, 0, s>>>(L.nbl, L.bnd_list.p, L.n, L.k, L.idx.p,
                                                                       L.A64.p, L.bnd_idx.p, L.bnd_A64.p,
                                                                       L.bnd_A32.p);
        MGM_LAUNCHED();
        // compact FP32-path indices
        {
            DBuf<int> ovf(3);
            ovf.zero(s);
            L.off16.alloc(nk4);
            k_make_offsets<<<blocks_for((long)nk4, 256), 256, 0, s>>>(L.n, L.ld4, L.k, L.sidx.p, nullptr, L.off16.p,
                                                                    ovf.p);
            MGM_LAUNCHED();
            if (l > 0) {
                const int kr = c->L[l - 1].k;
                L.r_off16.alloc((size_t)L.n * kr);
                k_make_offsets<<<blocks_for((long)L.n * kr, 256), 256, 0, s>>>(L.n, L.n, kr, L.s_r_idx.p, L.rpts.p,
                                                                             L.r_off16.p, ovf.p + 1);
                MGM_LAUNCHED();
            }
            if (l < c->nl - 1) {
                const int kp = c->L[l + 1].k;
                L.p_off16.alloc((size_t)L.n * kp);
                k_make_offsets<<<blocks_for((long)L.n * kp, 256), 256, 0, s>>>(L.n, L.n, kp, L.s_p_idx.p, L.ppts.p,
                                                                             L.p_off16.p, ovf.p + 2);
                MGM_LAUNCHED();
            }
            int h_ovf[3] = {0, 0, 0};
            ovf.download(h_ovf, 3, s);
            MGM_CUDA(cudaStreamSynchronize(s));
            L.off_ok = h_ovf[0] == 0;
            L.r_off_ok = h_ovf[1] == 0;
            L.p_off_ok = h_ovf[2] == 0;
        }
        // tile-streamed copy of the compact operator for the large levels
        L.ldt = 0;
        L.A32t.release();
        L.off16t.release();
        if (L.off_ok && L.n >= kTileMinRows && L.k <= kTileMaxK) {
            const int ld = (L.n + kTileRows - 1) / kTileRows * kTileRows;
            L.A32t.alloc((size_t)L.k * ld);
            L.off16t.alloc((size_t)L.k * ld);
            const long tot = (long)L.k * ld;
            k_tile_major<float><<<blocks_for(tot, 256), 256, 0, s>>>(L.n, L.k, ld, L.ld4, L.A32.p, L.A32t.p);
            MGM_LAUNCHED();
            k_tile_major<short><<<blocks_for(tot, 256), 256, 0, s>>>(L.n, L.k, ld, L.ld4, L.off16.p, L.off16t.p);
            MGM_LAUNCHED();
            L.ldt = ld;
        }
        // FP16 operator for the large levels
        L.W16.release();
        L.ldi = 0;
        L.h_ok = false;
        if (L.off_ok && L.n >= kVecMinRows) {
            const int ldi = (L.n + 127) / 128 * 128;
            DBuf<int> ovf(1);
            ovf.zero(s);
            L.W16.alloc((size_t)L.k * (ldi / 4));
            k_pack_half<<<blocks_for(ldi / 4, 256), 256, 0, s>>>(L.n, L.k, L.ld4, ldi, L.A32.p, L.off16.p,
                                                                L.dinv32.p, L.btag.p, L.W16.p, ovf.p);
            MGM_LAUNCHED();
            int h_ovf = 0;
            ovf.download(&h_ovf, 1, s);
            MGM_CUDA(cudaStreamSynchronize(s));
            L.h_ok = h_ovf == 0;
            L.ldi = ldi;
            if (!L.h_ok) L.W16.release();
        }
        for (DBuf<double> *b : {&L.p, &L.ptmp, &L.src, &L.res, &L.r64, &L.e64, &L.e64b, &L.d64, &L.q64}) { b->alloc(L.n); b->zero(s); }
        for (DBuf<float> *b : {&L.r32, &L.e32, &L.e32b, &L.d32, &L.q32}) { b->alloc(L.n); b->zero(s); }
    }
    {
        // the power iteration reads the operator in the level's own slot order
        const bool compact = c->compact;
        c->compact = false;
        for (int l = 0; l < c->nl - 1; l++) {
            auto lv = solve_levels<double>(c);
            estimate_lmax<double>(lv[l], s);
            c->L[l].lmax = lv[l].lmax;
        }
        c->compact = compact;
    }
    Level &Lc = c->L[c->nl - 1];
    MGM_REQUIRE(Lc.n <= 8192, "mgm_setup: coarsest level too large for the dense solve (use more levels)");
    c->cinv64.alloc((size_t)Lc.n * Lc.n);
    c->cinv32.alloc((size_t)Lc.n * Lc.n);
    dense_inverse(Lc.n, Lc.k, Lc.idx.p, Lc.A64.p, c->cinv64.p, c->cinv32.p, s);
    const int n0 = c->L[0].n;
    for (DBuf<double> *b : {&c->u, &c->v, &c->w, &c->u_new, &c->v_new, &c->w_new, &c->dpdn, &c->u_old, &c->v_old,
                            &c->w_old, &c->p_old, &c->dpdx, &c->dpdy, &c->dpdz, &c->tu, &c->tv, &c->tw}) {
        b->alloc(n0);
        b->zero(s);
    }
    c->partial.alloc(blocks_for(n0, 32) + 8);  // per-warp partial sums (k_correct)
    c->scal.alloc(8);
    c->tma_err.alloc(1);
    c->tma_err.zero(s);
    c->fused_bar.alloc(2);
    c->fused_bar.zero(s);
    c->fused_blocks = fused_vcycle_blocks();
    MGM_CUDA(cudaStreamSynchronize(s));
    if (!cooperative_in_conditional_ok(c)) c->fused_blocks = 0;  // the per-operation kernels then
    alloc_solver_buffers(c);
    MGM_CUDA(cudaStreamSynchronize(s));
    c->setup_done = true;
}

}  // namespace

extern "C" {

int mgm_setup(mgm_ctx *c, int flags)
{
    return guard([&] {
        check_ctx(c);
        for (int l = 0; l < c->nl; l++) MGM_REQUIRE(c->L[l].n > 0, "mgm_setup: level " + std::to_string(l) + " not set");
        c->setup_done = false;
        pipeline_geometry(c);
        c->have_ref_transfer = (flags & MGM_SETUP_REFERENCE_TRANSFER) != 0;
        pipeline_transfer(c, c->have_ref_transfer);
        pipeline_derivatives(c);
        prepare_solver(c);
    });
}

int mgm_load_level(mgm_ctx *c, int lev, int n, int nb, const double *x, const double *y, const double *z,
                   const double *nx, const double *ny, const double *nz, const unsigned char *btag, int poly_degree,
                   int k, const int *cloud, const double *Dx, const double *Dy, const double *Dz, const double *lap,
                   const double *lapP, const int *rpts, const int *ppts, double d_avg)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(lev >= 0 && lev < c->nl, "mgm_load_level: level out of range");
        MGM_REQUIRE(n > 0 && nb >= 0 && nb <= n && k >= 2 && k <= kMaxK, "mgm_load_level: bad sizes");
        MGM_REQUIRE(x && y && z && nx && ny && nz && btag && cloud && Dx && Dy && lap && lapP && rpts && ppts,
                    "mgm_load_level: null pointer");
        MGM_REQUIRE(c->dim == 2 || Dz, "mgm_load_level: Dz required in 3D");
        for (long t = 0; t < (long)n * k; t++) MGM_REQUIRE(cloud[t] >= 0 && cloud[t] < n, "mgm_load_level: cloud index out of range");
        Level &L = c->L[lev];
        L = Level();
        Monomials mono = monomials(c->dim, poly_degree);
        L.n = n; L.nb = nb; L.k = k; L.poly = poly_degree; L.np = mono.np; L.d_avg = d_avg;
        cudaStream_t s = c->s;
        L.x.upload(x, n, s); L.y.upload(y, n, s); L.z.upload(z, n, s);
        L.nx.upload(nx, n, s); L.ny.upload(ny, n, s); L.nz.upload(nz, n, s);
        L.btag.upload(btag, n, s);
        L.cloud.upload(cloud, (size_t)n * k, s);
        L.idx.alloc((size_t)n * k);
        transpose_rowmajor_to_ell_i(L.cloud.p, L.idx.p, n, k, s);
        const double *h[5] = {Dx, Dy, Dz, lap, lapP};
        DBuf<double> *dst[5] = {&L.Dx, &L.Dy, &L.Dz, &L.lap, &L.lapP};
        DBuf<double> tmp((size_t)n * k);
        for (int t = 0; t < 5; t++) {
            if (t == 2 && c->dim != 3) continue;
            tmp.upload(h[t], (size_t)n * k, s);
            dst[t]->alloc((size_t)n * k);
            transpose_rowmajor_to_ell_d(tmp.p, dst[t]->p, n, k, s);
            MGM_CUDA(cudaStreamSynchronize(s));
        }
        L.rpts.upload(rpts, n, s);
        L.ppts.upload(ppts, n, s);
        MGM_CUDA(cudaStreamSynchronize(s));
        c->setup_done = false;
        c->have_ref_transfer = false;
    });
}

int mgm_load_transfer(mgm_ctx *c, int lev, const double *restr, const double *prol)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(lev >= 0 && lev < c->nl && c->L[lev].n > 0, "mgm_load_transfer: level not loaded");
        Level &L = c->L[lev];
        cudaStream_t s = c->s;
        if (restr && lev > 0) {
            Level &F = c->L[lev - 1];
            DBuf<double> tmp;
            tmp.upload(restr, (size_t)L.n * F.k, s);
            L.ref_restr.alloc((size_t)L.n * F.k);
            transpose_rowmajor_to_ell_d(tmp.p, L.ref_restr.p, L.n, F.k, s);
            L.ref_r_idx.alloc((size_t)L.n * F.k);
            k_gather_idx<<<blocks_for((long)L.n * F.k, 256), 256, 0, s>>>(L.n, F.k, L.rpts.p, F.cloud.p, L.ref_r_idx.p);
            MGM_LAUNCHED();
            MGM_CUDA(cudaStreamSynchronize(s));
        }
        if (prol && lev < c->nl - 1) {
            Level &C = c->L[lev + 1];
            DBuf<double> tmp;
            tmp.upload(prol, (size_t)L.n * C.k, s);
            L.ref_prol.alloc((size_t)L.n * C.k);
            transpose_rowmajor_to_ell_d(tmp.p, L.ref_prol.p, L.n, C.k, s);
            L.ref_p_idx.alloc((size_t)L.n * C.k);
            k_gather_idx<<<blocks_for((long)L.n * C.k, 256), 256, 0, s>>>(L.n, C.k, L.ppts.p, C.cloud.p, L.ref_p_idx.p);
            MGM_LAUNCHED();
            MGM_CUDA(cudaStreamSynchronize(s));
        }
    });
}

int mgm_prepare(mgm_ctx *c)
{
    return guard([&] {
        check_ctx(c);
        for (int l = 0; l < c->nl; l++) MGM_REQUIRE(c->L[l].n > 0 && c->L[l].lapP.p, "mgm_prepare: level " + std::to_string(l) + " not loaded");
        bool ref_ok = true;
        for (int l = 0; l < c->nl; l++) {
            if (l > 0 && !c->L[l].ref_restr.p) ref_ok = false;
            if (l < c->nl - 1 && !c->L[l].ref_prol.p) ref_ok = false;
        }
        pipeline_transfer(c, false);
        c->have_ref_transfer = ref_ok;
        prepare_solver(c);
    });
}

int mgm_level_size(mgm_ctx *c, int lev, int *n, int *nb, int *k, int *np)
{
    return guard([&] {
        MGM_REQUIRE(c && lev >= 0 && lev < c->nl, "mgm_level_size: bad level");
        Level &L = c->L[lev];
        if (n) *n = L.n;
        if (nb) *nb = L.nb;
        if (k) *k = L.k;
        if (np) *np = L.np;
    });
}

int mgm_level_d_avg(mgm_ctx *c, int lev, double *d)
{
    return guard([&] {
        MGM_REQUIRE(c && lev >= 0 && lev < c->nl && c->setup_done, "mgm_level_d_avg: not set up");
        *d = c->L[lev].d_avg;
    });
}

int mgm_get_geometry(mgm_ctx *c, int lev, double *x, double *y, double *z, double *nx, double *ny, double *nz,
                     unsigned char *btag, int *cloud)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(lev >= 0 && lev < c->nl && c->setup_done, "mgm_get_geometry: not set up");
        Level &L = c->L[lev];
        cudaStream_t s = c->s;
        double *h[6] = {x, y, z, nx, ny, nz};
        DBuf<double> *d[6] = {&L.x, &L.y, &L.z, &L.nx, &L.ny, &L.nz};
        for (int t = 0; t < 6; t++) if (h[t]) d[t]->download(h[t], L.n, s);
        if (btag) L.btag.download(btag, L.n, s);
        if (cloud) L.cloud.download(cloud, (size_t)L.n * L.k, s);
        MGM_CUDA(cudaStreamSynchronize(s));
    });
}

int mgm_get_operators(mgm_ctx *c, int lev, double *Dx, double *Dy, double *Dz, double *lap, double *lapP)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(lev >= 0 && lev < c->nl && c->setup_done, "mgm_get_operators: not set up");
        Level &L = c->L[lev];
        cudaStream_t s = c->s;
        const size_t nk = (size_t)L.n * L.k;
        double *h[5] = {Dx, Dy, Dz, lap, lapP};
        DBuf<double> *d[5] = {&L.Dx, &L.Dy, &L.Dz, &L.lap, &L.lapP};
        DBuf<double> tmp(nk);
        for (int t = 0; t < 5; t++) {
            if (!h[t] || (t == 2 && c->dim != 3)) continue;
            transpose_ell_to_rowmajor_d(d[t]->p, tmp.p, L.n, L.k, s);
            tmp.download(h[t], nk, s);
            MGM_CUDA(cudaStreamSynchronize(s));
        }
    });
}

int mgm_get_transfer(mgm_ctx *c, int lev, int *rpts, int *ppts, double *restr, double *prol)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(lev >= 0 && lev < c->nl && c->setup_done, "mgm_get_transfer: not set up");
        Level &L = c->L[lev];
        cudaStream_t s = c->s;
        if (rpts) L.rpts.download(rpts, L.n, s);
        if (ppts) L.ppts.download(ppts, L.n, s);
        if (restr && lev > 0) {
            MGM_REQUIRE(c->have_ref_transfer, "mgm_get_transfer: reference transfer rows were not built");
            const int kf = c->L[lev - 1].k;
            DBuf<double> tmp((size_t)L.n * kf);
            transpose_ell_to_rowmajor_d(L.ref_restr.p, tmp.p, L.n, kf, s);
            tmp.download(restr, (size_t)L.n * kf, s);
            MGM_CUDA(cudaStreamSynchronize(s));
        }
        if (prol && lev < c->nl - 1) {
            MGM_REQUIRE(c->have_ref_transfer, "mgm_get_transfer: reference transfer rows were not built");
            const int kc = c->L[lev + 1].k;
            DBuf<double> tmp((size_t)L.n * kc);
            transpose_ell_to_rowmajor_d(L.ref_prol.p, tmp.p, L.n, kc, s);
            tmp.download(prol, (size_t)L.n * kc, s);
            MGM_CUDA(cudaStreamSynchronize(s));
        }
        MGM_CUDA(cudaStreamSynchronize(s));
    });
}

int mgm_get_solver_transfer(mgm_ctx *c, int lev, double *restr, double *prol)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(lev >= 0 && lev < c->nl && c->setup_done, "mgm_get_solver_transfer: not set up");
        Level &L = c->L[lev];
        cudaStream_t s = c->s;
        if (restr && lev > 0) {
            const int kf = c->L[lev - 1].k;
            DBuf<double> tmp((size_t)L.n * kf);
            transpose_ell_to_rowmajor_d(L.s_r_w64.p, tmp.p, L.n, kf, s);
            tmp.download(restr, (size_t)L.n * kf, s);
            MGM_CUDA(cudaStreamSynchronize(s));
        }
        if (prol && lev < c->nl - 1) {
            const int kc = c->L[lev + 1].k;
            DBuf<double> tmp((size_t)L.n * kc);
            transpose_ell_to_rowmajor_d(L.s_p_w64.p, tmp.p, L.n, kc, s);
            tmp.download(prol, (size_t)L.n * kc, s);
            MGM_CUDA(cudaStreamSynchronize(s));
        }
    });
}

int mgm_get_compact(mgm_ctx *c, int lev, int which, int *idx, float *w, int *compact)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(lev >= 0 && lev < c->nl && c->setup_done, "mgm_get_compact: not set up");
        MGM_REQUIRE(which >= 0 && which <= 2, "mgm_get_compact: which must be 0, 1 or 2");
        MGM_REQUIRE(idx && w, "mgm_get_compact: null output");
        MGM_REQUIRE(which != 1 || lev > 0, "mgm_get_compact: level 0 has no restriction into it");
        MGM_REQUIRE(which != 2 || lev < c->nl - 1, "mgm_get_compact: the coarsest level has no prolongation into it");
        Level &L = c->L[lev];
        cudaStream_t s = c->s;
        int k = L.k, ld = L.ld4;
        const short *off = nullptr;
        const int *base = nullptr, *gidx = nullptr;
        const float *W = nullptr;
        if (which == 0) {
            off = L.off_ok ? L.off16.p : nullptr; gidx = L.sidx.p; W = L.A32.p;
        } else if (which == 1) {
            k = c->L[lev - 1].k; ld = L.n;
            off = L.r_off_ok ? L.r_off16.p : nullptr; base = L.rpts.p; gidx = L.s_r_idx.p; W = L.s_r_w32.p;
        } else {
            k = c->L[lev + 1].k; ld = L.n;
            off = L.p_off_ok ? L.p_off16.p : nullptr; base = L.ppts.p; gidx = L.s_p_idx.p; W = L.s_p_w32.p;
        }
        const size_t nk = (size_t)L.n * k;
        DBuf<int> di(nk);
        DBuf<float> dw(nk);
        k_decode_compact<<<blocks_for((long)nk, 256), 256, 0, s>>>(L.n, k, ld, off, base, gidx, W, di.p, dw.p);
        MGM_LAUNCHED();
        di.download(idx, nk, s);
        dw.download(w, nk, s);
        MGM_CUDA(cudaStreamSynchronize(s));
        if (compact) *compact = off ? 1 : 0;
    });
}

int mgm_set_flow(mgm_ctx *c, double Re, double courant, float omega, int num_relax, int num_vcycles, double dt)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done, "mgm_set_flow: call mgm_setup first");
        MGM_REQUIRE(Re > 0 && num_relax >= 0 && num_vcycles >= 0, "mgm_set_flow: bad parameters");
        c->Re = Re; c->courant = courant; c->omega = omega; c->num_relax = num_relax; c->num_vcycles = num_vcycles;
        c->rho = 1;
        const double mu = c->rho / Re;
        c->nu = mu / c->rho;
        if (dt > 0) c->dt = dt;
        else {
            // calculate_dt (general_functions.h:34-41)
            const double d = c->L[0].d_avg;
            const double termd = 2 * c->nu / (d * d);
            const double termc = 1 / d;
            c->dt = 0.5 / (termd + termc) * courant;
        }
    });
}

int mgm_get_dt(mgm_ctx *c, double *dt)
{
    return guard([&] { MGM_REQUIRE(c, "null context"); *dt = c->dt; });
}

static DBuf<double> *field_buf(mgm_ctx *c, int lev, int which)
{
    Level &L = c->L[lev];
    if (lev == 0) {
        switch (which) {
        case MGM_FIELD_U: return &c->u;
        case MGM_FIELD_V: return &c->v;
        case MGM_FIELD_W: return &c->w;
        case MGM_FIELD_U_NEW: return &c->u_new;
        case MGM_FIELD_V_NEW: return &c->v_new;
        case MGM_FIELD_W_NEW: return &c->w_new;
        case MGM_FIELD_DPDN: return &c->dpdn;
        case MGM_FIELD_U_OLD: return &c->u_old;
        case MGM_FIELD_V_OLD: return &c->v_old;
        case MGM_FIELD_W_OLD: return &c->w_old;
        case MGM_FIELD_DPDX: return &c->dpdx;
        case MGM_FIELD_DPDY: return &c->dpdy;
        case MGM_FIELD_DPDZ: return &c->dpdz;
        case MGM_FIELD_P_OLD: return &c->p_old;
        }
    }
    switch (which) {
    case MGM_FIELD_P: return &L.p;
    case MGM_FIELD_RES: return &L.res;
    case MGM_FIELD_SOURCE: return &L.src;
    }
    throw Error{MGM_ERR_ARG, "unknown field id for this level"};
}

int mgm_set_field(mgm_ctx *c, int lev, int which, const double *values)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done && lev >= 0 && lev < c->nl, "mgm_set_field: not set up");
        field_buf(c, lev, which)->upload(values, c->L[lev].n, c->s);
        MGM_CUDA(cudaStreamSynchronize(c->s));
    });
}

int mgm_get_field(mgm_ctx *c, int lev, int which, double *values)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done && lev >= 0 && lev < c->nl, "mgm_get_field: not set up");
        field_buf(c, lev, which)->download(values, c->L[lev].n, c->s);
        MGM_CUDA(cudaStreamSynchronize(c->s));
    });
}

int mgm_apply_bc(mgm_ctx *c, int kind)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done, "mgm_apply_bc: call mgm_setup first");
        MGM_REQUIRE(kind == MGM_BC_LID || kind == MGM_BC_TAYLOR_COUETTE, "mgm_apply_bc: unknown kind");
        cudaStream_t s = c->s;
        // every field starts from zero, as the reference's calloc'd fields do
        for (DBuf<double> *b : {&c->u, &c->v, &c->w, &c->u_new, &c->v_new, &c->w_new, &c->u_old, &c->v_old,
                                &c->w_old, &c->dpdn, &c->dpdx, &c->dpdy, &c->dpdz, &c->p_old})
            b->zero(s);
        for (int l = 0; l < c->nl; l++) {
            c->L[l].p.zero(s);
            c->L[l].src.zero(s);
            c->L[l].res.zero(s);
        }
        c->hist_ok.zero(s);  // no pressure history from rest
        Level &L = c->L[0];
        k_bc<<<blocks_for(L.n, 256), 256, 0, s>>>(L.n, kind, L.x.p, L.y.p, c->u.p, c->v.p, c->u_new.p, c->v_new.p);
        MGM_LAUNCHED();
        MGM_CUDA(cudaStreamSynchronize(s));
    });
}

int mgm_set_solver(mgm_ctx *c, double rel_tol, int max_iters, int cheb_degree, double cheb_ratio)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(rel_tol > 0 && max_iters >= 1 && max_iters <= kMaxKrylov && cheb_degree >= 1 && cheb_degree <= 16 &&
                        cheb_ratio > 1, "mgm_set_solver: bad parameters");
        MGM_CUDA(cudaStreamSynchronize(c->s));
        drop_graphs(c);
        c->tol = rel_tol; c->cheb_deg = cheb_degree; c->cheb_ratio = cheb_ratio;
        if (max_iters != c->max_iters) {
            c->max_iters = max_iters;
            if (c->setup_done) alloc_solver_buffers(c);
        }
    });
}

int mgm_ref_routine(mgm_ctx *c, int level, int routine)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done, "mgm_ref_routine: not ready");
        MGM_REQUIRE(c->have_ref_transfer || c->nl == 1,
                    "mgm_ref_routine: needs mgm_setup(..., MGM_SETUP_REFERENCE_TRANSFER) or mgm_load_transfer");
        const bool pair = routine == MGM_REF_RESTRICT || routine == MGM_REF_PROLONGATE;
        MGM_REQUIRE(level >= 0 && level < c->nl - (pair ? 1 : 0), "mgm_ref_routine: level out of range");
        auto R = ref_levels(c);
        const double w1 = (double)c->omega, w2 = (double)(1 - c->omega);
        switch (routine) {
        case MGM_REF_RELAXATION: ref_relaxation(R[level], w1, w2, c->num_relax, c->s); break;
        case MGM_REF_RESIDUALS: ref_residual_interior(R[level], c->s); break;
        case MGM_REF_RESTRICT: ref_restrict(R[level], R[level + 1], c->s); break;
        case MGM_REF_PROLONGATE: ref_prolongate(R[level], R[level + 1], c->s); break;
        default: throw Error{MGM_ERR_ARG, "mgm_ref_routine: unknown routine"};
        }
        MGM_CUDA(cudaStreamSynchronize(c->s));
    });
}

int mgm_use_compact(mgm_ctx *c, int enable)
{
    return guard([&] {
        check_ctx(c);
        MGM_CUDA(cudaStreamSynchronize(c->s));
        drop_graphs(c);
        c->compact = enable != 0;
    });
}

int mgm_use_tiled(mgm_ctx *c, int enable)
{
    return guard([&] {
        check_ctx(c);
        MGM_CUDA(cudaStreamSynchronize(c->s));
        drop_graphs(c);
        c->use_tma = enable != 0;
    });
}

int mgm_set_compatible_rhs(mgm_ctx *c, int enable)
{
    return guard([&] {
        check_ctx(c);
        c->compat = enable != 0;
        if (c->compat && c->setup_done) ensure_compat(c);
    });
}

int mgm_use_half_operator(mgm_ctx *c, int enable)
{
    return guard([&] {
        check_ctx(c);
        MGM_CUDA(cudaStreamSynchronize(c->s));
        drop_graphs(c);
        c->half_operator = enable != 0;
    });
}

int mgm_use_fused_coarse(mgm_ctx *c, int enable)
{
    return guard([&] {
        check_ctx(c);
        MGM_CUDA(cudaStreamSynchronize(c->s));
        drop_graphs(c);
        c->fused_coarse = enable != 0;
    });
}

int mgm_selftest_barrier_timeout(mgm_ctx *c, int *status)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(status, "mgm_selftest_barrier_timeout: null argument");
        MGM_CUDA(cudaSetDevice(c->device));
        cudaStream_t s = c->s;
        MGM_CUDA(cudaStreamSynchronize(s));
        c->tma_err.zero(s);
        c->fused_bar.zero(s);
        MGM_CUDA(launch_barrier_selftest(s, c->fused_bar.p, c->tma_err.p));
        MGM_LAUNCHED();
        *status = MGM_OK;
        try {
            check_wait_flags(c, s);  // clears the flags and the barrier when the wait ran out
        } catch (const Error &e) {
            *status = e.code;
        }
    });
}

int mgm_fused_coarse_available(mgm_ctx *c, int *available)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(available, "mgm_fused_coarse_available: null argument");
        *available = c->fused_blocks > 0 ? 1 : 0;
    });
}

int mgm_use_launch_chaining(mgm_ctx *c, int enable)
{
    return guard([&] {
        check_ctx(c);
        MGM_CUDA(cudaStreamSynchronize(c->s));
        drop_graphs(c);
        c->chain_launches = enable != 0;
    });
}

int mgm_use_graphs(mgm_ctx *c, int enable)
{
    return guard([&] {
        check_ctx(c);
        MGM_CUDA(cudaStreamSynchronize(c->s));
        drop_graphs(c);
        c->use_graphs = enable != 0;
    });
}

int mgm_use_step_graph(mgm_ctx *c, int enable)
{
    return guard([&] {
        check_ctx(c);
        MGM_CUDA(cudaStreamSynchronize(c->s));
        drop_step_graphs(c);
        c->step_graphs = enable != 0;
    });
}

int mgm_solve_counters(mgm_ctx *c, long long *vcycles, long long *cycles, long long *solves)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done && c->fg.p, "mgm_solve_counters: not set up");
        const FgState &h = read_fg_head(c);
        if (vcycles) *vcycles = h.vcycles_total;
        if (cycles) *cycles = h.cycles_total;
        if (solves) *solves = h.solves_total;
    });
}

int mgm_solve_start_residual(mgm_ctx *c, double *geo_mean)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done && c->fg.p && geo_mean, "mgm_solve_start_residual: not set up");
        const FgState &h = read_fg_head(c);
        *geo_mean = h.solves_total > 0 ? std::pow(10.0, h.start_log_relres / (double)h.solves_total) : 0.0;
    });
}

int mgm_set_initial_guess(mgm_ctx *c, int flags)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE((flags & ~(MGM_GUESS_EXTRAPOLATE | MGM_GUESS_LEARNED)) == 0, "mgm_set_initial_guess: unknown flag");
        MGM_REQUIRE(!(flags & MGM_GUESS_LEARNED) || (c->mpnn != nullptr),
                    "mgm_set_initial_guess: the learned guess needs a network (mgm_mpnn_init)");
        c->guess_flags = flags;
    });
}

int mgm_set_warm_smoothing(mgm_ctx *c, int steps)
{
    return guard([&] {
        MGM_REQUIRE(c && steps >= 0 && steps <= 16, "mgm_set_warm_smoothing: 0..16 steps");
        c->warm_smooth_steps = steps;
    });
}

int mgm_last_learned_alpha(mgm_ctx *c, double *alpha)
{
    return guard([&] {
        MGM_REQUIRE(c, "null context");
        *alpha = c->last_learned_alpha;
    });
}

int mgm_last_solve(mgm_ctx *c, int *iters, double *rel_res)
{
    return guard([&] {
        MGM_REQUIRE(c, "null context");
        if (iters) *iters = c->last_iters;
        if (rel_res) *rel_res = c->last_relres;
    });
}

int mgm_intermediate_velocity(mgm_ctx *c)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done && c->dt > 0, "mgm_intermediate_velocity: call mgm_setup and mgm_set_flow first");
        launch_momentum(step_args(c), c->dim, c->s);
        MGM_CUDA(cudaStreamSynchronize(c->s));
    });
}

int mgm_mass_residual(mgm_ctx *c)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done && c->dt > 0, "mgm_mass_residual: not ready");
        launch_divergence(step_args(c), c->dim, c->s);
        MGM_CUDA(cudaStreamSynchronize(c->s));
    });
}

int mgm_poisson(mgm_ctx *c, int mode)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done, "mgm_poisson: not ready");
        poisson(c, mode);
        MGM_CUDA(cudaStreamSynchronize(c->s));
    });
}

int mgm_update_velocity(mgm_ctx *c, double *mass_res)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done && c->dt > 0, "mgm_update_velocity: not ready");
        StepArgs a = step_args(c);
        launch_correct(a, c->dim, c->partial.p, c->scal.p, c->s);
        if (mass_res) {
            launch_mass_diag(a, c->dim, c->partial.p, c->scal.p + 1, c->s);
            c->scal.download(c->h_pinned, 2, c->s);
            MGM_CUDA(cudaStreamSynchronize(c->s));
            *mass_res = c->h_pinned[1];
        }
        MGM_CUDA(cudaStreamSynchronize(c->s));
    });
}

int mgm_last_steady_error(mgm_ctx *c, double *steady_err)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done, "mgm_last_steady_error: not ready");
        c->scal.download(c->h_pinned, 1, c->s);
        MGM_CUDA(cudaStreamSynchronize(c->s));
        *steady_err = c->h_pinned[0];
    });
}

int mgm_step(mgm_ctx *c, int mode, double *steady_err)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done && c->dt > 0, "mgm_step: call mgm_setup and mgm_set_flow first");
        const double e = step_timed(c, mode);
        if (steady_err) *steady_err = e;
    });
}

int mgm_run_steps(mgm_ctx *c, int mode, int nsteps, double *step_ms, double *poisson_ms, long long *vcycles,
                  double *steady_err)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done && c->dt > 0, "mgm_run_steps: call mgm_setup and mgm_set_flow first");
        MGM_REQUIRE(nsteps >= 0, "mgm_run_steps: nsteps < 0");
        ensure_events(c);
        prepare_steps(c, mode);
        if (step_graph_usable(c, mode)) step_graph(c, mode);  // captured before the timed region
        fg_clear_totals(c->fg.p, c->s);
        c->ref_vcycles_acc = 0;
        MGM_CUDA(cudaEventRecord(c->ev[0], c->s));
        const double e = run_steps_device(c, mode, nsteps);
        MGM_CUDA(cudaEventRecord(c->ev[1], c->s));
        MGM_CUDA(cudaEventSynchronize(c->ev[1]));
        float ms = 0;
        MGM_CUDA(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
        const FgState &h = read_fg_head(c);
        if (step_ms) *step_ms = ms;
        if (poisson_ms) *poisson_ms = h.t_ns * 1e-6;
        if (vcycles) *vcycles = mode == MGM_MODE_REFERENCE ? c->ref_vcycles_acc : h.vcycles_total;
        if (steady_err) *steady_err = e;
    });
}

int mgm_step_host(mgm_ctx *c, int mode, const double *u_in, const double *v_in, const double *w_in, double *u_out,
                  double *v_out, double *w_out, double *p_out, double *steady_err)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done && c->dt > 0, "mgm_step_host: call mgm_setup and mgm_set_flow first");
        const size_t nb = sizeof(double) * c->L[0].n;
        cudaStream_t s = c->s;
        if (u_in) MGM_CUDA(cudaMemcpyAsync(c->u.p, u_in, nb, cudaMemcpyHostToDevice, s));
        if (v_in) MGM_CUDA(cudaMemcpyAsync(c->v.p, v_in, nb, cudaMemcpyHostToDevice, s));
        if (w_in) MGM_CUDA(cudaMemcpyAsync(c->w.p, w_in, nb, cudaMemcpyHostToDevice, s));
        const double e = step_timed(c, mode);
        if (u_out) MGM_CUDA(cudaMemcpyAsync(u_out, c->u.p, nb, cudaMemcpyDeviceToHost, s));
        if (v_out) MGM_CUDA(cudaMemcpyAsync(v_out, c->v.p, nb, cudaMemcpyDeviceToHost, s));
        if (w_out) MGM_CUDA(cudaMemcpyAsync(w_out, c->w.p, nb, cudaMemcpyDeviceToHost, s));
        if (p_out) MGM_CUDA(cudaMemcpyAsync(p_out, c->L[0].p.p, nb, cudaMemcpyDeviceToHost, s));
        MGM_CUDA(cudaStreamSynchronize(s));
        if (steady_err) *steady_err = e;
    });
}

void *mgm_host_alloc(size_t bytes)
{
    void *p = nullptr;
    int st = guard([&] { MGM_CUDA(cudaMallocHost(&p, bytes)); });
    return st == MGM_OK ? p : nullptr;
}

void mgm_host_free(void *p)
{
    if (p) cudaFreeHost(p);
}

int mgm_profile_smoother(mgm_ctx *c, int enable)
{
    return guard([&] {
        check_ctx(c);
        MGM_CUDA(cudaStreamSynchronize(c->s));
        c->prof.harvest();
        drop_graphs(c);
        c->prof.used = 0;
        c->prof.on = enable != 0;
        c->prof.ms = 0;
        c->prof.launches = 0;
    });
}

int mgm_profile_read(mgm_ctx *c, double *ms_total, long long *launches, long long *bytes_per_launch)
{
    return guard([&] {
        check_ctx(c);
        MGM_CUDA(cudaStreamSynchronize(c->s));
        if (ms_total) *ms_total = c->prof.ms;
        if (launches) *launches = c->prof.launches;
        if (bytes_per_launch) {
            // level-0 Chebyshev step of MGM_MODE_FP32_IR, each array counted once:
            // per slot the weight and the index (FP32 + int16, FP16 + int16 on the
            // half-precision operator, FP32 + int32 on the plain layout); per node
            // r, dinv, e read, e' written, d written, d read by all but the first
            // step of a smoothing pass, btag
            const Level &L = c->L[0];
            const bool compact = c->compact && L.off_ok;
            const bool half = compact && c->half_operator && L.h_ok && !(c->use_tma && L.ldt > 0);
            const double slot = half ? 4.0 : compact ? 6.0 : 8.0;
            const double dread = 4.0 * (c->cheb_deg - 1) / (double)c->cheb_deg;
            *bytes_per_launch = (long long)((double)L.n * (L.k * slot + 4 * 5 + 1 + dread));
        }
    });
}

int mgm_solve_poisson(mgm_ctx *c, int mode, const double *b, double *p, int *iters, double *rel_res)
{
    return guard([&] {
        check_ctx(c);
        MGM_REQUIRE(c->setup_done, "mgm_solve_poisson: not ready");
        MGM_REQUIRE(mode == MGM_MODE_FP64 || mode == MGM_MODE_FP32_IR, "mgm_solve_poisson: mode must be FP64 or FP32_IR");
        Level &L0 = c->L[0];
        L0.src.upload(b, L0.n, c->s);
        L0.p.upload(p, L0.n, c->s);
        poisson(c, mode);
        L0.p.download(p, L0.n, c->s);
        MGM_CUDA(cudaStreamSynchronize(c->s));
        if (iters) *iters = c->last_iters;
        if (rel_res) *rel_res = c->last_relres;
    });
}

int mgm_sync(mgm_ctx *c)
{
    return guard([&] {
        check_ctx(c);
        MGM_CUDA(cudaStreamSynchronize(c->s));
    });
}

}  // extern "C"
