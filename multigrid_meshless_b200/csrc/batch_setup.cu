// batch_setup.cu -- set-up of a hierarchy whose stencil size varies per node,
// with every per-node saddle-point system of every level (derivative rows,
// restriction rows, prolongation rows) solved in ONE persistent launch.
//
// Systems have uneven orders N = k_i + np (k_i from the node's level and
// distance to the boundary, np from the level's polynomial degree).  The host
// sorts them by N (largest first), cuts each size class into tiles of g
// systems, and the persistent kernel's CTAs pull tiles from a global counter.
// Inside a CTA each of the g systems of a tile is solved by a team of
// 256/g threads in its own shared-memory slot, synchronised by a named
// barrier.  An autotuner picks, per size class, the team width, and for the
// launch the shared-memory budget per CTA (hence CTAs per SM), by timing the
// same kernel on samples of each class.
//
// The arithmetic of each system is that of the fixed-stencil kernels
// (weights.cuh), i.e. of rbf.h:42-421 and mesh_functions.h:533-670; the
// stencil of node i is the first k_i entries of its nearest-node list.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "batch.cuh"

namespace mgm {

struct BLevelDev {
    int n, kmax;
    const double *x, *y, *z, *nx, *ny, *nz;
    const uint8_t *btag;
    const int *kk, *cloud, *rp;
    double *Dx, *Dy, *Dz, *lap, *lapP;
    const int *rpts, *ppts, *r_rp, *p_rp;
    double *r_w, *p_w;
    MonoDev mono;
};

__constant__ BLevelDev c_blev[kBatchMaxLevels];
__constant__ int c_bdim, c_bphs;

struct WTask {
    int code;  // level | kind << 4 ; kind 0 derivative row, 1 restriction row, 2 prolongation row
    int row;
};

// One system, solved by team tm in the shared-memory slot `slot`.
__device__ void solve_system(const Team &tm, WTask task, double *slot)
{
    const int dim = c_bdim, phs = c_bphs;
    const int lev = task.code & 15, kind = task.code >> 4, i = task.row;
    const BLevelDev &T = c_blev[lev];
    const BLevelDev &S = c_blev[kind == 0 ? lev : (kind == 1 ? lev - 1 : lev + 1)];
    const int ip = kind == 0 ? i : (kind == 1 ? T.rpts[i] : T.ppts[i]);
    const int m = S.kk[ip], np = S.mono.np, N = m + np;
    double *aug = slot;
    double *sx = aug + (size_t)2 * N * N, *sy = sx + m, *sz = sy + m;
    double *L = sz + m;     // [4][N]
    double *t = L + 4 * N;  // [N]
    double *wout = t + N;   // [4][m]
    int *perm = (int *)(wout + 4 * m);
    stage_cloud(tm, S.cloud + (long)ip * S.kmax, m, S.x, S.y, S.z, sx, sy, sz);
    tm.sync();
    build_aug(tm, m, np, dim, phs, S.mono, sx, sy, sz, aug, N);
    const int nops = dim == 3 ? 4 : 3;
    if (kind == 0) {
        for (int o = 0; o < nops; o++)
            operator_row0(tm, o == nops - 1 ? 3 : o, m, np, dim, phs, S.mono, sx, sy, sz, L + o * N);
    } else {
        const double p1[3] = {T.x[i], T.y[i], T.z[i]};
        const double seed[3] = {S.x[ip], S.y[ip], S.z[ip]};
        transfer_row(tm, m, np, dim, phs, S.mono, sx, sy, sz, p1, seed, L);
    }
    tm.sync();
    gauss_jordan(tm, aug, perm, t, N);
    if (kind == 0) {
        for (int e = tm.tid; e < nops * m; e += tm.size) {
            const int o = e / m, j = e % m;
            wout[o * m + j] = row_times_inverse(L + o * N, aug, perm, N, j);
        }
        tm.sync();
        const long base = T.rp[i];
        const bool bnd = T.btag[i] != 0;
        const double nxi = T.nx[i], nyi = T.ny[i], nzi = T.nz[i];
        for (int j = tm.tid; j < m; j += tm.size) {
            const double dx = wout[j], dy = wout[m + j], dl = wout[(nops - 1) * m + j];
            T.Dx[base + j] = dx;
            T.Dy[base + j] = dy;
            T.lap[base + j] = dl;
            double dz = 0;
            if (dim == 3) { dz = wout[2 * m + j]; T.Dz[base + j] = dz; }
            if (bnd) {
                double v = MGM_ADD(MGM_MUL(dx, nxi), MGM_MUL(dy, nyi));
                if (dim == 3) v = MGM_ADD(v, MGM_MUL(dz, nzi));
                T.lapP[base + j] = v;
            } else T.lapP[base + j] = dl;
        }
    } else {
        double *W = kind == 1 ? T.r_w : T.p_w;
        const long base = kind == 1 ? T.r_rp[i] : T.p_rp[i];
        for (int j = tm.tid; j < m; j += tm.size) W[base + j] = row_times_inverse(L, aug, perm, N, j);
    }
    tm.sync();  // the slot is reused by the team's next system
}

// tiles[t] = {first task, systems in the tile, threads per system, slot bytes}
__global__ void __launch_bounds__(kBatchCta) k_weights_persistent(const int4 *__restrict__ tiles, int ntiles,
                                                                  const WTask *__restrict__ tasks, int *counter)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ int cur;
    for (;;) {
        if (threadIdx.x == 0) cur = atomicAdd(counter, 1);
        __syncthreads();
        const int t = cur;
        if (t >= ntiles) break;
        const int4 tile = tiles[t];
        const int team = tile.z, grp = threadIdx.x / team;
        if (grp < tile.y) {
            const Team tm{(int)threadIdx.x % team, team, team == kBatchCta ? 0 : 1 + grp};
            solve_system(tm, tasks[tile.x + grp], (double *)(smraw + (size_t)grp * tile.w));
        }
        __syncthreads();
    }
}

// CSR columns: row i takes the first len(i) entries of src_cloud[src[i]] (src = nullptr: row i itself)
__global__ void k_prefix_cols(int nrows, const int *__restrict__ rp, const int *__restrict__ src,
                              const int *__restrict__ src_cloud, int src_kmax, int *__restrict__ col)
{
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= nrows) return;
    const int beg = rp[w], len = rp[w + 1] - beg;
    const int s = src ? src[w] : w;
    for (int j = lane; j < len; j += 32) col[beg + j] = src_cloud[(long)s * src_kmax + j];
}

namespace {

int num_sms()
{
    int dev = 0, v = 0;
    MGM_CUDA(cudaGetDevice(&dev));
    MGM_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
    return std::max(1, v);
}

void upload_level_table(mgm_batch *b)
{
    BLevelDev d[kBatchMaxLevels];
    std::memset(d, 0, sizeof(d));
    for (int l = 0; l < b->nl; l++) {
        BLevel &L = b->L[l];
        BLevelDev &o = d[l];
        o.n = L.n; o.kmax = L.kmax;
        o.x = L.x.p; o.y = L.y.p; o.z = L.z.p; o.nx = L.nx.p; o.ny = L.ny.p; o.nz = L.nz.p;
        o.btag = L.btag.p; o.kk = L.kk.p; o.cloud = L.cloud.p; o.rp = L.rp.p;
        o.Dx = L.Dx.p; o.Dy = L.Dy.p; o.Dz = L.Dz.p; o.lap = L.lap.p; o.lapP = L.lapP.p;
        o.rpts = L.rpts.p; o.ppts = L.ppts.p; o.r_rp = L.r_rp.p; o.p_rp = L.p_rp.p;
        o.r_w = L.r_w64.p; o.p_w = L.p_w64.p;
        o.mono = to_dev(monomials(b->dim, L.poly));
    }
    MGM_CUDA(cudaMemcpyToSymbolAsync(c_blev, d, sizeof(d), 0, cudaMemcpyHostToDevice, b->s));
    MGM_CUDA(cudaMemcpyToSymbolAsync(c_bdim, &b->dim, sizeof(int), 0, cudaMemcpyHostToDevice, b->s));
    MGM_CUDA(cudaMemcpyToSymbolAsync(c_bphs, &b->phs, sizeof(int), 0, cudaMemcpyHostToDevice, b->s));
}

// kNN lists with k_max entries, breadth-first reorder, normals, CSR structure
void level_geometry(mgm_batch *b, int l)
{
    BLevel &L = b->L[l];
    cudaStream_t s = b->s;
    const int n = L.n, nb = L.nb, km = L.kmax;
    L.cloud.alloc((size_t)n * km);
    GridIndex gall, gint;
    grid_build(gall, n, L.x.p, L.y.p, L.z.p, nullptr, b->dim, s);
    if (n > nb)
        knn_query(gall, L.x.p, L.y.p, L.z.p, n - nb, L.x.p + nb, L.y.p + nb, L.z.p + nb, nullptr, km, 0,
                  L.cloud.p + (size_t)nb * km, km, s);
    if (nb > 0) {
        grid_build(gint, n, L.x.p, L.y.p, L.z.p, L.btag.p, b->dim, s);
        knn_query(gint, L.x.p, L.y.p, L.z.p, nb, L.x.p, L.y.p, L.z.p, nullptr, km, 1, L.cloud.p, km, s);
    }
    DBuf<int> q1(n);
    const int reached = bfs_order(n, km, L.cloud.p, q1.p, s);
    MGM_REQUIRE(reached == n, "mgm_batch_setup: stencil graph of level " + std::to_string(l) + " is disconnected");
    apply_order(n, km, q1.p, L.x.p, L.y.p, L.z.p, L.nx.p, L.ny.p, L.nz.p, L.btag.p, L.cloud.p, s);
    correct_normals(n, km, L.x.p, L.y.p, L.z.p, L.btag.p, L.cloud.p, L.nx.p, L.ny.p, L.nz.p, s);
    std::vector<int> hq(n);
    q1.download(hq.data(), n, s);
    MGM_CUDA(cudaStreamSynchronize(s));
    std::vector<int> kk(n);
    for (int i = 0; i < n; i++) kk[i] = L.h_kk[hq[i]];
    L.h_kk.swap(kk);
    L.kk.upload(L.h_kk.data(), n, s);
    std::vector<int> rp(n + 1, 0);
    long long acc = 0;
    for (int i = 0; i < n; i++) { rp[i] = (int)acc; acc += L.h_kk[i]; }
    MGM_REQUIRE(acc < (1LL << 31), "mgm_batch_setup: too many stencil entries on one level");
    rp[n] = (int)acc;
    L.nnz = acc;
    L.rp.upload(rp.data(), n + 1, s);
    L.col.alloc((size_t)std::max<long long>(acc, 1));
    k_prefix_cols<<<blocks_for((long)n * 32, 256), 256, 0, s>>>(n, L.rp.p, nullptr, L.cloud.p, km, L.col.p);
    MGM_LAUNCHED();
    for (DBuf<double> *o : {&L.Dx, &L.Dy, &L.lap, &L.lapP}) o->alloc((size_t)std::max<long long>(acc, 1));
    if (b->dim == 3) L.Dz.alloc((size_t)std::max<long long>(acc, 1));
}

void nearest(const BLevel &T, const BLevel &S, int dim, DBuf<int> &out, cudaStream_t s)
{
    GridIndex g;
    grid_build(g, S.n, S.x.p, S.y.p, S.z.p, nullptr, dim, s);
    out.alloc(T.n);
    knn_query(g, S.x.p, S.y.p, S.z.p, T.n, T.x.p, T.y.p, T.z.p, nullptr, 1, 0, out.p, 1, s);
}

// CSR structure of a transfer matrix whose row i interpolates from the cloud of src[i]
long long transfer_structure(const std::vector<int> &src, const std::vector<uint8_t> &skip, const BLevel &S,
                             DBuf<int> &rp_d, DBuf<int> &col_d, const DBuf<int> &src_d, cudaStream_t s)
{
    const int nt = (int)src.size();
    std::vector<int> rp(nt + 1);
    long long acc = 0;
    for (int i = 0; i < nt; i++) { rp[i] = (int)acc; if (!skip[i]) acc += S.h_kk[src[i]]; }
    MGM_REQUIRE(acc < (1LL << 31), "mgm_batch_setup: too many transfer entries");
    rp[nt] = (int)acc;
    rp_d.upload(rp.data(), nt + 1, s);
    col_d.alloc((size_t)std::max<long long>(acc, 1));
    k_prefix_cols<<<blocks_for((long)nt * 32, 256), 256, 0, s>>>(nt, rp_d.p, src_d.p, S.cloud.p, S.kmax, col_d.p);
    MGM_LAUNCHED();
    return acc;
}

struct Budget {
    int smem = 0;  // dynamic shared memory per CTA
    int ctas = 0;  // resident CTAs per SM at that size
};

std::vector<Budget> budgets()
{
    int dev = 0, optin = 0;
    MGM_CUDA(cudaGetDevice(&dev));
    MGM_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa;
    MGM_CUDA(cudaFuncGetAttributes(&fa, k_weights_persistent));
    const int cap = (optin - (int)fa.sharedSizeBytes) & ~15;  // opt-in maximum less the static shared memory
    MGM_CUDA(cudaFuncSetAttribute(k_weights_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize, cap));
    std::vector<Budget> out;
    for (int want = 1; want <= 4; want++) {
        int smem = std::min(cap, (233472 / want - 1024 - 64) & ~15);
        for (int tries = 0; tries < 64 && smem > 0; tries++) {
            int occ = 0;
            MGM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_weights_persistent, kBatchCta, smem));
            if (occ >= want) break;
            smem -= 1024;
        }
        int occ = 0;
        MGM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_weights_persistent, kBatchCta, smem));
        if (occ >= want && (out.empty() || occ > out.back().ctas)) out.push_back(Budget{smem, occ});
    }
    MGM_REQUIRE(!out.empty(), "mgm_batch_setup: the weight kernel cannot be resident");
    return out;
}

// tiles of g systems over tasks[first, first + count)
void make_tiles(std::vector<int4> &tiles, long long first, long long count, int g, int slot)
{
    for (long long q = 0; q < count; q += g)
        tiles.push_back(make_int4((int)(first + q), (int)std::min<long long>(g, count - q), kBatchCta / g, slot));
}

double run_tiles(const std::vector<int4> &tiles, const WTask *d_tasks, int smem, int grid, cudaStream_t s)
{
    if (tiles.empty()) return 0.0;
    DBuf<int4> dt;
    dt.upload(tiles.data(), tiles.size(), s);
    DBuf<int> counter(1);
    counter.zero(s);
    cudaEvent_t e0, e1;
    MGM_CUDA(cudaEventCreate(&e0));
    MGM_CUDA(cudaEventCreate(&e1));
    MGM_CUDA(cudaEventRecord(e0, s));
    k_weights_persistent<<<std::max(1, std::min<int>(grid, (int)tiles.size())), kBatchCta, smem, s>>>(
        dt.p, (int)tiles.size(), d_tasks, counter.p);
    MGM_LAUNCHED();
    MGM_CUDA(cudaEventRecord(e1, s));
    MGM_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    MGM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms;
}

}  // namespace

void batch_setup(mgm_batch *b, bool autotune)
{
    cudaStream_t s = b->s;
    for (int l = 0; l < b->nl; l++) {
        BLevel &L = b->L[l];
        MGM_REQUIRE(L.n > 0, "mgm_batch_setup: level " + std::to_string(l) + " not set");
        L.np = monomials(b->dim, L.poly).np;
        for (int kv : L.h_kk) MGM_REQUIRE(system_bytes(kv, L.np) <= 232448, "mgm_batch_setup: system too large for shared memory");
        level_geometry(b, l);
    }
    for (int l = 0; l < b->nl; l++) {
        BLevel &L = b->L[l];
        nearest(L, l < b->nl - 1 ? b->L[l + 1] : L, b->dim, L.ppts, s);
        nearest(L, l > 0 ? b->L[l - 1] : L, b->dim, L.rpts, s);
    }
    MGM_CUDA(cudaStreamSynchronize(s));
    // transfer structures (restriction: non-boundary rows except the pinned node; prolongation: every row)
    std::vector<std::vector<int>> h_rpts(b->nl), h_ppts(b->nl);
    std::vector<std::vector<uint8_t>> h_btag(b->nl);
    for (int l = 0; l < b->nl; l++) {
        BLevel &L = b->L[l];
        h_rpts[l].resize(L.n); h_ppts[l].resize(L.n); h_btag[l].resize(L.n);
        L.rpts.download(h_rpts[l].data(), L.n, s);
        L.ppts.download(h_ppts[l].data(), L.n, s);
        L.btag.download(h_btag[l].data(), L.n, s);
    }
    MGM_CUDA(cudaStreamSynchronize(s));
    for (int l = 0; l < b->nl; l++) {
        BLevel &L = b->L[l];
        L.nb = 0;
        for (uint8_t t : h_btag[l]) L.nb += t != 0;
        if (l > 0) {
            std::vector<uint8_t> skip(L.n);
            for (int i = 0; i < L.n; i++) skip[i] = h_btag[l][i] != 0 || i == 0;
            L.r_nnz = transfer_structure(h_rpts[l], skip, b->L[l - 1], L.r_rp, L.r_col, L.rpts, s);
            L.r_w64.alloc((size_t)std::max<long long>(L.r_nnz, 1));
            L.r_w64.zero(s);
        }
        if (l < b->nl - 1) {
            std::vector<uint8_t> skip(L.n, 0);
            L.p_nnz = transfer_structure(h_ppts[l], skip, b->L[l + 1], L.p_rp, L.p_col, L.ppts, s);
            L.p_w64.alloc((size_t)std::max<long long>(L.p_nnz, 1));
        }
    }
    upload_level_table(b);
    // task list, bucketed by system order N (largest first)
    std::vector<std::vector<WTask>> bucket(kMaxN + 1);
    std::vector<int> max_m(kMaxN + 1, 0);
    auto add = [&](int code, int row, int m, int np) {
        const int N = m + np;
        MGM_REQUIRE(N <= kMaxN && m >= 2, "mgm_batch_setup: stencil size out of range");
        bucket[N].push_back(WTask{code, row});
        max_m[N] = std::max(max_m[N], m);
    };
    for (int l = 0; l < b->nl; l++) {
        BLevel &L = b->L[l];
        for (int i = 0; i < L.n; i++) add(l, i, L.h_kk[i], L.np);
        if (l > 0) {
            const BLevel &F = b->L[l - 1];
            for (int i = 0; i < L.n; i++)
                if (!(h_btag[l][i] != 0 || i == 0)) add(l | (1 << 4), i, F.h_kk[h_rpts[l][i]], F.np);
        }
        if (l < b->nl - 1) {
            const BLevel &C = b->L[l + 1];
            for (int i = 0; i < L.n; i++) add(l | (2 << 4), i, C.h_kk[h_ppts[l][i]], C.np);
        }
    }
    std::vector<WTask> tasks;
    std::vector<std::pair<long long, long long>> span(kMaxN + 1, {0, 0});  // first, count per N
    for (int N = kMaxN; N >= 1; N--) {
        span[N] = {(long long)tasks.size(), (long long)bucket[N].size()};
        tasks.insert(tasks.end(), bucket[N].begin(), bucket[N].end());
        std::vector<WTask>().swap(bucket[N]);
    }
    b->systems = (long long)tasks.size();
    DBuf<WTask> d_tasks;
    d_tasks.upload(tasks.data(), tasks.size(), s);
    const int sms = num_sms();
    const std::vector<Budget> bud = budgets();
    // per budget and class: best team width
    const int gs[4] = {1, 2, 4, 8};
    std::vector<int> Ns;
    for (int N = kMaxN; N >= 1; N--) if (span[N].second > 0) Ns.push_back(N);
    int best_b = -1;
    double best_total = 1e300;
    std::vector<std::vector<int>> choice(bud.size(), std::vector<int>(kMaxN + 1, 0));
    std::vector<std::vector<double>> us(bud.size(), std::vector<double>(kMaxN + 1, 0.0));
    b->tuning_ms = 0;
    for (size_t bi = 0; bi < bud.size(); bi++) {
        double total = 0;
        bool feasible = true;
        for (int N : Ns) {
            const size_t need = system_bytes(max_m[N], N - max_m[N]);
            int gbest = 0;
            double tbest = 1e300;
            for (int g : gs) {
                const int slot = (bud[bi].smem / g) & ~15;
                if ((size_t)slot < need) break;
                if (!autotune) { gbest = g; if (g >= 4) break; continue; }
                const long long count = span[N].second;
                const long long sample = std::min<long long>(count, (long long)sms * bud[bi].ctas * g * 2);
                std::vector<int4> tl;
                make_tiles(tl, span[N].first, sample, g, slot);
                const double ms = run_tiles(tl, d_tasks.p, bud[bi].smem, sms * bud[bi].ctas, s);
                b->tuning_ms += ms;
                const double per = ms * 1e3 / (double)sample;
                if (per < tbest) { tbest = per; gbest = g; }
            }
            if (gbest == 0) { feasible = false; break; }
            choice[bi][N] = gbest;
            us[bi][N] = autotune ? tbest : 0.0;
            total += autotune ? tbest * (double)span[N].second : 0.0;
        }
        if (!feasible) continue;
        if (!autotune) {
            // without tuning: the budget with two CTAs per SM if every class fits, else the largest
            if (best_b < 0 || bud[bi].ctas == 2) best_b = (int)bi;
            continue;
        }
        if (total < best_total) { best_total = total; best_b = (int)bi; }
    }
    MGM_REQUIRE(best_b >= 0, "mgm_batch_setup: no shared-memory budget fits every system");
    const Budget &B = bud[best_b];
    std::vector<int4> tiles;
    b->classes.clear();
    for (int N : Ns) {
        const int g = choice[best_b][N];
        make_tiles(tiles, span[N].first, span[N].second, g, (B.smem / g) & ~15);
        BatchClass c;
        c.N = N; c.count = span[N].second; c.team = kBatchCta / g; c.us_per_system = us[best_b][N];
        b->classes.push_back(c);
    }
    b->tiles = (int)tiles.size();
    b->smem_bytes = B.smem;
    b->ctas_per_sm = B.ctas;
    b->weights_ms = run_tiles(tiles, d_tasks.p, B.smem, sms * B.ctas, s);
    batch_prepare_solver(b);
    b->setup_done = true;
}

}  // namespace mgm
