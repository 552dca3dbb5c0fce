// setup.cu -- sm_100a kernels of the per-level set-up pipeline:
//   grid-hash kNN clouds        (kdtree_functions.h:61-175)
//   breadth-first reordering    (mesh_functions.h:774-872)
//   normals, average spacing    (mesh_functions.h:478-527, 895-910)
//   batched FP64 saddle-point weight solves (rbf.h:42-421, mat_lib.h:423-491,
//                                mesh_functions.h:533-670)
#include <algorithm>
#include <cfloat>
#include <climits>

#include "mgm_internal.cuh"
#include "weights.cuh"

namespace mgm {

// ===========================================================================
// exclusive scan (three-phase, recursive over block sums)
// ===========================================================================
constexpr int SCAN_BS = 256, SCAN_PT = 8, SCAN_TILE = SCAN_BS * SCAN_PT;

__global__ void k_scan_tile(const int *__restrict__ in, int *__restrict__ out, int n, int *__restrict__ sums)
{
    __shared__ int s[SCAN_BS];
    long base = (long)blockIdx.x * SCAN_TILE + (long)threadIdx.x * SCAN_PT;
    int v[SCAN_PT], t = 0;
#pragma unroll
    for (int i = 0; i < SCAN_PT; i++) { long idx = base + i; v[i] = idx < n ? in[idx] : 0; t += v[i]; }
    s[threadIdx.x] = t;
    __syncthreads();
    for (int off = 1; off < SCAN_BS; off <<= 1) {
        int a = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
        __syncthreads();
        s[threadIdx.x] += a;
        __syncthreads();
    }
    int run = s[threadIdx.x] - t;
#pragma unroll
    for (int i = 0; i < SCAN_PT; i++) { long idx = base + i; if (idx < n) out[idx] = run; run += v[i]; }
    if (threadIdx.x == SCAN_BS - 1) sums[blockIdx.x] = s[SCAN_BS - 1];
}

__global__ void k_scan_add(int *__restrict__ out, int n, const int *__restrict__ offs)
{
    long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < n) out[idx] += offs[idx / SCAN_TILE];
}

__global__ void k_scan_total(const int *in, const int *out, int n, int *total)
{
    *total = n > 0 ? out[n - 1] + in[n - 1] : 0;
}

static void scan_rec(const int *d_in, int *d_out, int n, cudaStream_t s)
{
    int nb = blocks_for(n, SCAN_TILE);
    int *sums = nullptr, *sums_scan = nullptr;
    MGM_CUDA(cudaMallocAsync(&sums, sizeof(int) * (size_t)std::max(nb, 1), s));
    MGM_CUDA(cudaMallocAsync(&sums_scan, sizeof(int) * (size_t)std::max(nb, 1), s));
    k_scan_tile<<<nb, SCAN_BS, 0, s>>>(d_in, d_out, n, sums);
    MGM_LAUNCHED();
    if (nb > 1) {
        scan_rec(sums, sums_scan, nb, s);
        k_scan_add<<<blocks_for(n, 256), 256, 0, s>>>(d_out, n, sums_scan);
        MGM_LAUNCHED();
    }
    MGM_CUDA(cudaFreeAsync(sums, s));
    MGM_CUDA(cudaFreeAsync(sums_scan, s));
}

void scan_exclusive(const int *d_in, int *d_out, int n, int *d_total, cudaStream_t s)
{
    if (n > 0) scan_rec(d_in, d_out, n, s);
    if (d_total) {
        k_scan_total<<<1, 1, 0, s>>>(d_in, d_out, n, d_total);
        MGM_LAUNCHED();
    }
}

// ===========================================================================
// grid hash
// ===========================================================================
__global__ void k_bbox(int n, const double *x, const double *y, const double *z, const uint8_t *mask, double *part)
{
    // part[block*7 + {0..5}] = xmin,xmax,ymin,ymax,zmin,zmax ; [6] = count
    __shared__ double s[6][256];
    __shared__ int sc[256];
    double v[6] = {DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX};
    int c = 0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        if (mask && mask[i]) continue;
        c++;
        v[0] = fmin(v[0], x[i]); v[1] = fmax(v[1], x[i]);
        v[2] = fmin(v[2], y[i]); v[3] = fmax(v[3], y[i]);
        v[4] = fmin(v[4], z[i]); v[5] = fmax(v[5], z[i]);
    }
    for (int q = 0; q < 6; q++) s[q][threadIdx.x] = v[q];
    sc[threadIdx.x] = c;
    __syncthreads();
    for (int off = blockDim.x / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            for (int q = 0; q < 6; q += 2) {
                s[q][threadIdx.x] = fmin(s[q][threadIdx.x], s[q][threadIdx.x + off]);
                s[q + 1][threadIdx.x] = fmax(s[q + 1][threadIdx.x], s[q + 1][threadIdx.x + off]);
            }
            sc[threadIdx.x] += sc[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int q = 0; q < 6; q++) part[blockIdx.x * 7 + q] = s[q][0];
        part[blockIdx.x * 7 + 6] = (double)sc[0];
    }
}

struct GridDev {
    int dim, ncx, ncy, ncz;
    double x0, y0, z0, inv_cell, cell;
};

__device__ __forceinline__ int grid_cell_of(const GridDev &g, double px, double py, double pz, int &cx, int &cy, int &cz)
{
    cx = (int)floor((px - g.x0) * g.inv_cell);
    cy = (int)floor((py - g.y0) * g.inv_cell);
    cz = g.dim == 3 ? (int)floor((pz - g.z0) * g.inv_cell) : 0;
    cx = min(max(cx, 0), g.ncx - 1);
    cy = min(max(cy, 0), g.ncy - 1);
    cz = min(max(cz, 0), g.ncz - 1);
    return (cz * g.ncy + cy) * g.ncx + cx;
}

__global__ void k_grid_count(int n, const double *x, const double *y, const double *z, const uint8_t *mask, GridDev g,
                             int *cid, int *counts)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (mask && mask[i]) { cid[i] = -1; return; }
    int cx, cy, cz;
    int c = grid_cell_of(g, x[i], y[i], z[i], cx, cy, cz);
    cid[i] = c;
    atomicAdd(&counts[c], 1);
}

__global__ void k_grid_fill(int n, const int *cid, int *fill, int *items)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = cid[i];
    if (c < 0) return;
    int pos = atomicAdd(&fill[c], 1);
    items[pos] = (int)i;
}

void grid_build(GridIndex &g, int n, const double *dx, const double *dy, const double *dz, const uint8_t *dmask, int dim,
                cudaStream_t s)
{
    const int nbk = std::min(blocks_for(n, 256), 1184);
    DBuf<double> part((size_t)std::max(nbk, 1) * 7);
    k_bbox<<<std::max(nbk, 1), 256, 0, s>>>(n, dx, dy, dz, dmask, part.p);
    MGM_LAUNCHED();
    std::vector<double> hp((size_t)std::max(nbk, 1) * 7);
    part.download(hp.data(), hp.size(), s);
    MGM_CUDA(cudaStreamSynchronize(s));
    double b[6] = {DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX};
    long cnt = 0;
    for (int i = 0; i < std::max(nbk, 1); i++) {
        for (int q = 0; q < 6; q += 2) { b[q] = std::min(b[q], hp[i * 7 + q]); b[q + 1] = std::max(b[q + 1], hp[i * 7 + q + 1]); }
        cnt += (long)hp[i * 7 + 6];
    }
    if (cnt == 0) { for (int q = 0; q < 6; q++) b[q] = 0; }
    double ex = std::max(b[1] - b[0], 1e-300), ey = std::max(b[3] - b[2], 1e-300), ez = std::max(b[5] - b[4], 1e-300);
    double per = dim == 3 ? 2.0 : 2.0;  // ~2 nodes per cell
    double cell = dim == 3 ? cbrt(per * ex * ey * ez / std::max(cnt, 1L)) : sqrt(per * ex * ey / std::max(cnt, 1L));
    if (!(cell > 0) || !std::isfinite(cell)) cell = 1.0;
    g.dim = dim; g.cell = cell; g.x0 = b[0]; g.y0 = b[2]; g.z0 = b[4];
    // cap the cell count so that degenerate (flat) extents cannot explode the table
    auto cells_along = [&](double e) { return (int)std::min(e / cell, 1.0e6) + 1; };
    g.ncx = cells_along(b[1] - b[0]); g.ncy = cells_along(b[3] - b[2]); g.ncz = dim == 3 ? cells_along(b[5] - b[4]) : 1;
    long nc = (long)g.ncx * g.ncy * g.ncz;
    MGM_REQUIRE(nc < (1L << 30), "grid hash: cell table too large");
    GridDev gd{g.dim, g.ncx, g.ncy, g.ncz, g.x0, g.y0, g.z0, 1.0 / g.cell, g.cell};
    DBuf<int> cid(std::max(n, 1)), counts(nc);
    counts.zero(s);
    g.start.alloc(nc + 1);
    g.items.alloc(std::max(cnt, 1L));
    k_grid_count<<<blocks_for(n, 256), 256, 0, s>>>(n, dx, dy, dz, dmask, gd, cid.p, counts.p);
    MGM_LAUNCHED();
    scan_exclusive(counts.p, g.start.p, (int)nc, g.start.p + nc, s);
    DBuf<int> fill(nc);
    MGM_CUDA(cudaMemcpyAsync(fill.p, g.start.p, sizeof(int) * nc, cudaMemcpyDeviceToDevice, s));
    k_grid_fill<<<blocks_for(n, 256), 256, 0, s>>>(n, cid.p, fill.p, g.items.p);
    MGM_LAUNCHED();
    MGM_CUDA(cudaStreamSynchronize(s));
}

// One thread per query: rings of cells around the query's cell are scanned
// until the k-th best distance is below the distance at which unscanned cells
// begin.  Candidates are ranked by (distance, node index).
__global__ void __launch_bounds__(128) k_knn(GridDev g, const int *__restrict__ start, const int *__restrict__ items,
                                             const double *__restrict__ px, const double *__restrict__ py,
                                             const double *__restrict__ pz, int nq, const double *__restrict__ qx,
                                             const double *__restrict__ qy, const double *__restrict__ qz,
                                             const int *__restrict__ self_id, int k, int mode, int *__restrict__ out,
                                             int ld)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const int want = mode == 1 ? k - 1 : k;
    double bd[kMaxK];
    int bi[kMaxK];
    int have = 0;
    const double x = qx[q], y = qy[q], z = qz[q];
    int cx, cy, cz;
    grid_cell_of(g, x, y, z, cx, cy, cz);
    const int rmax = g.ncx + g.ncy + g.ncz;
    for (int r = 0; r <= rmax && want > 0; r++) {
        const int zlo = g.dim == 3 ? cz - r : 0, zhi = g.dim == 3 ? cz + r : 0;
        for (int zz = max(zlo, 0); zz <= min(zhi, g.ncz - 1); zz++) {
            const int dz = abs(zz - cz);
            for (int yy = max(cy - r, 0); yy <= min(cy + r, g.ncy - 1); yy++) {
                const int dyv = abs(yy - cy);
                const bool full_row = (dz == r) || (dyv == r);
                for (int xx = max(cx - r, 0); xx <= min(cx + r, g.ncx - 1); xx += 1) {
                    if (!full_row && abs(xx - cx) != r) {
                        // jump to the other side of the ring in this row
                        if (xx < cx + r) { xx = cx + r - 1; continue; }
                    }
                    const int c = (zz * g.ncy + yy) * g.ncx + xx;
                    for (int t = start[c]; t < start[c + 1]; t++) {
                        const int p = items[t];
                        const double d = mgm_ref_distance(x, y, z, px[p], py[p], pz[p]);
                        if (have == want && (d > bd[want - 1] || (d == bd[want - 1] && p > bi[want - 1]))) continue;
                        int pos = have < want ? have : want - 1;
                        while (pos > 0 && (bd[pos - 1] > d || (bd[pos - 1] == d && bi[pos - 1] > p))) {
                            bd[pos] = bd[pos - 1];
                            bi[pos] = bi[pos - 1];
                            pos--;
                        }
                        bd[pos] = d;
                        bi[pos] = p;
                        if (have < want) have++;
                    }
                }
            }
        }
        // unscanned cells start at least r cells away (a small margin covers the
        // rounding of the cell assignment of points near cell faces)
        if (have == want && bd[want - 1] < ((double)r - 1e-3) * g.cell) break;
    }
    int *row = out + (long)q * ld;
    if (mode == 1) {
        row[0] = self_id ? self_id[q] : q;
        for (int j = 0; j < want; j++) row[1 + j] = j < have ? bi[j] : 0;
    } else {
        for (int j = 0; j < want; j++) row[j] = j < have ? bi[j] : 0;
    }
}

void knn_query(const GridIndex &g, const double *px, const double *py, const double *pz, int nq, const double *qx,
               const double *qy, const double *qz, const int *self_id, int k, int mode, int *out, int ld, cudaStream_t s)
{
    MGM_REQUIRE(k >= 1 && k <= kMaxK, "kNN: k out of range");
    if (nq <= 0) return;
    GridDev gd{g.dim, g.ncx, g.ncy, g.ncz, g.x0, g.y0, g.z0, 1.0 / g.cell, g.cell};
    k_knn<<<blocks_for(nq, 128), 128, 0, s>>>(gd, g.start.p, g.items.p, px, py, pz, nq, qx, qy, qz, self_id, k, mode,
                                              out, ld);
    MGM_LAUNCHED();
}

// ===========================================================================
// breadth-first reordering: level-synchronous BFS that reproduces the FIFO
// order exactly.  A node discovered in level L+1 is appended in the order of
// the smallest (parent queue position, cloud slot) that reaches it.
// ===========================================================================
__global__ void k_bfs_claim(const int *__restrict__ cloud, int k, const int *__restrict__ queue, int head, int fsize,
                            const uint8_t *__restrict__ visited, int *__restrict__ key)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long total = (long)fsize * (k - 1);
    if (t >= total) return;
    int p = (int)(t / (k - 1)), j = 1 + (int)(t % (k - 1));
    int nb = cloud[(long)queue[head + p] * k + j];
    if (!visited[nb]) atomicMin(&key[nb], p * k + j);
}

__global__ void k_bfs_flag(const int *__restrict__ cloud, int k, const int *__restrict__ queue, int head, int fsize,
                           const uint8_t *__restrict__ visited, const int *__restrict__ key, int *__restrict__ flag)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long total = (long)fsize * (k - 1);
    if (t >= total) return;
    int p = (int)(t / (k - 1)), j = 1 + (int)(t % (k - 1));
    int nb = cloud[(long)queue[head + p] * k + j];
    flag[t] = (!visited[nb] && key[nb] == p * k + j) ? 1 : 0;
}

__global__ void k_bfs_append(const int *__restrict__ cloud, int k, int *__restrict__ queue, int head, int fsize, int tail,
                             uint8_t *__restrict__ visited, const int *__restrict__ flag, const int *__restrict__ pos)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long total = (long)fsize * (k - 1);
    if (t >= total || !flag[t]) return;
    int p = (int)(t / (k - 1)), j = 1 + (int)(t % (k - 1));
    int nb = cloud[(long)queue[head + p] * k + j];
    queue[tail + pos[t]] = nb;
    visited[nb] = 1;
}

__global__ void k_bfs_init(int n, int *key, uint8_t *visited, int *queue)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { key[i] = INT_MAX; visited[i] = i == 0; }
    if (i == 0) queue[0] = 0;
}

int bfs_order(int n, int k, const int *d_cloud, int *d_queue1, cudaStream_t s)
{
    MGM_REQUIRE(n >= 1 && k >= 2, "bfs_order: bad sizes");
    DBuf<int> key(n);
    DBuf<uint8_t> visited(n);
    k_bfs_init<<<blocks_for(n, 256), 256, 0, s>>>(n, key.p, visited.p, d_queue1);
    MGM_LAUNCHED();
    int head = 0, tail = 1;
    DBuf<int> flag, pos, total(1);
    int *h_total = nullptr;
    MGM_CUDA(cudaMallocHost(&h_total, sizeof(int)));
    try {
        while (head < tail) {
            int fsize = tail - head;
            long items = (long)fsize * (k - 1);
            MGM_REQUIRE(items < INT_MAX, "bfs_order: frontier too large");
            if ((long)flag.n < items) { flag.alloc(items); pos.alloc(items); }
            int nbk = blocks_for(items, 256);
            k_bfs_claim<<<nbk, 256, 0, s>>>(d_cloud, k, d_queue1, head, fsize, visited.p, key.p);
            MGM_LAUNCHED();
            k_bfs_flag<<<nbk, 256, 0, s>>>(d_cloud, k, d_queue1, head, fsize, visited.p, key.p, flag.p);
            MGM_LAUNCHED();
            scan_exclusive(flag.p, pos.p, (int)items, total.p, s);
            k_bfs_append<<<nbk, 256, 0, s>>>(d_cloud, k, d_queue1, head, fsize, tail, visited.p, flag.p, pos.p);
            MGM_LAUNCHED();
            MGM_CUDA(cudaMemcpyAsync(h_total, total.p, sizeof(int), cudaMemcpyDeviceToHost, s));
            MGM_CUDA(cudaStreamSynchronize(s));
            head = tail;
            tail += *h_total;
            MGM_REQUIRE(tail <= n, "bfs_order: queue overflow (corrupt cloud indices)");
        }
    } catch (...) {
        cudaFreeHost(h_total);
        throw;
    }
    cudaFreeHost(h_total);
    return tail;
}

__global__ void k_inverse_perm(int n, const int *q1, int *q2)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) q2[q1[i]] = (int)i;
}

template <class T>
__global__ void k_gather(int n, const int *q1, const T *in, T *out)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = in[q1[i]];
}

__global__ void k_gather_cloud(int n, int k, const int *q1, const int *q2, const int *in, int *out)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)n * k) return;
    long i = t / k;
    int j = (int)(t % k);
    out[t] = q2[in[(long)q1[i] * k + j]];
}

void apply_order(int n, int k, const int *q1, double *x, double *y, double *z, double *nx, double *ny, double *nz,
                 uint8_t *btag, int *cloud, cudaStream_t s)
{
    DBuf<int> q2(n), tc((size_t)n * k);
    DBuf<double> tmp(n);
    DBuf<uint8_t> tb(n);
    k_inverse_perm<<<blocks_for(n, 256), 256, 0, s>>>(n, q1, q2.p);
    MGM_LAUNCHED();
    double *arrs[6] = {x, y, z, nx, ny, nz};
    for (double *a : arrs) {
        k_gather<double><<<blocks_for(n, 256), 256, 0, s>>>(n, q1, a, tmp.p);
        MGM_LAUNCHED();
        MGM_CUDA(cudaMemcpyAsync(a, tmp.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    }
    k_gather<uint8_t><<<blocks_for(n, 256), 256, 0, s>>>(n, q1, btag, tb.p);
    MGM_LAUNCHED();
    MGM_CUDA(cudaMemcpyAsync(btag, tb.p, n, cudaMemcpyDeviceToDevice, s));
    k_gather_cloud<<<blocks_for((long)n * k, 256), 256, 0, s>>>(n, k, q1, q2.p, cloud, tc.p);
    MGM_LAUNCHED();
    MGM_CUDA(cudaMemcpyAsync(cloud, tc.p, sizeof(int) * (size_t)n * k, cudaMemcpyDeviceToDevice, s));
    MGM_CUDA(cudaStreamSynchronize(s));
}

// correct_normal_directions (mesh_functions.h:478-527)
__global__ void k_correct_normals(int n, int k, const double *x, const double *y, const double *z, const uint8_t *btag,
                                  const int *cloud, double *nx, double *ny, double *nz)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !btag[i]) return;
    double xa = 0, ya = 0, za = 0;
    int count = 0;
    for (int j = k - 1; j > 0; j--) {
        int c = cloud[i * k + j];
        if (!btag[c]) { xa = MGM_ADD(xa, x[c]); ya = MGM_ADD(ya, y[c]); za = MGM_ADD(za, z[c]); count = 1; break; }
    }
    double cd = (double)count;
    xa = MGM_DIV(xa, cd); ya = MGM_DIV(ya, cd); za = MGM_DIV(za, cd);
    double dx = MGM_SUB(xa, x[i]), dy = MGM_SUB(ya, y[i]), dz = MGM_SUB(za, z[i]);
    double a = nx[i], b = ny[i], c = nz[i];
    double dot = MGM_ADD(MGM_ADD(MGM_MUL(dx, a), MGM_MUL(dy, b)), MGM_MUL(dz, c));
    if (dot > 0) { a = -a; b = -b; c = -c; }
    double mag = MGM_SQRT(MGM_ADD(MGM_ADD(MGM_MUL(a, a), MGM_MUL(b, b)), MGM_MUL(c, c)));
    nx[i] = MGM_DIV(a, mag); ny[i] = MGM_DIV(b, mag); nz[i] = MGM_DIV(c, mag);
}

void correct_normals(int n, int k, const double *x, const double *y, const double *z, const uint8_t *btag,
                     const int *cloud, double *nx, double *ny, double *nz, cudaStream_t s)
{
    k_correct_normals<<<blocks_for(n, 256), 256, 0, s>>>(n, k, x, y, z, btag, cloud, nx, ny, nz);
    MGM_LAUNCHED();
}

// calculate_avg_dx (mesh_functions.h:895-910): the per-node lengths in
// parallel, then the sum in node order (the reference's rounding sequence).
__global__ void k_spacing(int n, int k, int dim, const double *x, const double *y, const double *z, const uint8_t *btag,
                          const int *cloud, double *len)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (btag[i]) { len[i] = 0.0; return; }
    int c = cloud[i * k + 1];
    double dx = MGM_SUB(x[i], x[c]), dy = MGM_SUB(y[i], y[c]), dz = dim == 3 ? MGM_SUB(z[i], z[c]) : 0.0;
    len[i] = MGM_SQRT(MGM_ADD(MGM_ADD(MGM_MUL(dx, dx), MGM_MUL(dy, dy)), MGM_MUL(dz, dz)));
}

__global__ void k_ordered_sum(int n, const double *len, double *out)
{
    // single thread: adding +0.0 for boundary nodes leaves the running sum unchanged
    double s = 0;
    int i = 0;
    for (; i + 8 <= n; i += 8) {
        double v0 = len[i], v1 = len[i + 1], v2 = len[i + 2], v3 = len[i + 3];
        double v4 = len[i + 4], v5 = len[i + 5], v6 = len[i + 6], v7 = len[i + 7];
        s = MGM_ADD(s, v0); s = MGM_ADD(s, v1); s = MGM_ADD(s, v2); s = MGM_ADD(s, v3);
        s = MGM_ADD(s, v4); s = MGM_ADD(s, v5); s = MGM_ADD(s, v6); s = MGM_ADD(s, v7);
    }
    for (; i < n; i++) s = MGM_ADD(s, len[i]);
    *out = MGM_DIV(s, (double)n);
}

void avg_dx(int n, int k, int dim, const double *x, const double *y, const double *z, const uint8_t *btag,
            const int *cloud, double *d_out, cudaStream_t s)
{
    DBuf<double> len(n);
    k_spacing<<<blocks_for(n, 256), 256, 0, s>>>(n, k, dim, x, y, z, btag, cloud, len.p);
    MGM_LAUNCHED();
    k_ordered_sum<<<1, 1, 0, s>>>(n, len.p, d_out);
    MGM_LAUNCHED();
    MGM_CUDA(cudaStreamSynchronize(s));
}

// ===========================================================================
// batched saddle-point weights: one CTA per node, the augmented [A | I]
// system of order N = k + np staged in shared memory, Gauss-Jordan with the
// reference's single bubble pass on column 0 and no further pivoting
// (mat_lib.h:423-491), every product/difference rounded separately.
// ===========================================================================
Monomials monomials(int dim, int deg)
{
    Monomials m;
    int c = 0;
    if (dim == 2) {
        for (int i = 0; i <= deg; i++)
            for (int j = 0; j <= deg - i; j++) { MGM_REQUIRE(c < kMaxPoly, "poly degree too high"); m.px[c] = i; m.py[c] = j; m.pz[c] = 0; c++; }
    } else {
        for (int i = 0; i <= deg; i++)
            for (int j = 0; j <= deg - i; j++)
                for (int l = 0; l <= deg - i - j; l++) { MGM_REQUIRE(c < kMaxPoly, "poly degree too high"); m.px[c] = i; m.py[c] = j; m.pz[c] = l; c++; }
    }
    m.np = c;
    return m;
}

__global__ void k_derivative_weights(int n, int k, int dim, int phs, MonoDev mono, const double *__restrict__ x,
                                     const double *__restrict__ y, const double *__restrict__ z,
                                     const double *__restrict__ nx, const double *__restrict__ ny,
                                     const double *__restrict__ nz, const uint8_t *__restrict__ btag,
                                     const int *__restrict__ cloud, double *Dx, double *Dy, double *Dz, double *lap,
                                     double *lapP)
{
    extern __shared__ double sm[];
    const int m = k, np = mono.np, N = m + np;
    double *aug = sm;
    double *sx = aug + (size_t)N * 2 * N, *sy = sx + m, *sz = sy + m;
    double *L = sz + m;           // [4][N]
    double *t = L + 4 * N;        // [N]
    double *wout = t + N;         // [4][k]
    int *perm = (int *)(wout + 4 * k);
    const int nops = dim == 3 ? 4 : 3;
    const Team tm = Team::block();
    for (long node = blockIdx.x; node < n; node += gridDim.x) {
        const int *cl = cloud + node * k;
        stage_cloud(tm, cl, m, x, y, z, sx, sy, sz);
        tm.sync();
        build_aug(tm, m, np, dim, phs, mono, sx, sy, sz, aug, N);
        for (int o = 0; o < nops; o++) operator_row0(tm, o == nops - 1 ? 3 : o, m, np, dim, phs, mono, sx, sy, sz, L + o * N);
        tm.sync();
        gauss_jordan(tm, aug, perm, t, N);
        // weights: D[j] = sum_c L[c] * inverse[c][j], c ascending (multiply_matrices, mat_lib.h:214-228)
        for (int e = threadIdx.x; e < nops * m; e += blockDim.x) {
            const int o = e / m, j = e % m;
            wout[o * k + j] = row_times_inverse(L + o * N, aug, perm, N, j);
        }
        __syncthreads();
        const bool bnd = btag[node] != 0;
        const double nxi = nx[node], nyi = ny[node], nzi = nz[node];
        for (int j = threadIdx.x; j < m; j += blockDim.x) {
            const long o = node * k + j;
            const double dx = wout[j], dy = wout[k + j], dl = wout[(nops - 1) * k + j];
            Dx[o] = dx; Dy[o] = dy; lap[o] = dl;
            double dz = 0;
            if (dim == 3) { dz = wout[2 * k + j]; Dz[o] = dz; }
            if (bnd) {
                double v = MGM_ADD(MGM_MUL(dx, nxi), MGM_MUL(dy, nyi));
                if (dim == 3) v = MGM_ADD(v, MGM_MUL(dz, nzi));
                lapP[o] = v;
            } else lapP[o] = dl;
        }
        __syncthreads();
    }
}

static size_t weights_smem(int k, int np) { return system_bytes(k, np); }

static int weights_grid(long rows)
{
    return (int)std::min<long>(rows, 148L * 64);
}

void derivative_weights(int n, int k, int dim, int phs, const Monomials &mono, const double *x, const double *y,
                        const double *z, const double *nx, const double *ny, const double *nz, const uint8_t *btag,
                        const int *cloud, double *Dx, double *Dy, double *Dz, double *lap, double *lapP, cudaStream_t s)
{
    MGM_REQUIRE(k >= 2 && k <= kMaxK && k + mono.np <= kMaxN, "weights: stencil too large");
    if (n <= 0) return;
    size_t smem = weights_smem(k, mono.np);
    MGM_REQUIRE(smem <= 227 * 1024, "weights: system does not fit in shared memory");
    MGM_CUDA(cudaFuncSetAttribute(k_derivative_weights, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_derivative_weights<<<weights_grid(n), 128, smem, s>>>(n, k, dim, phs, to_dev(mono), x, y, z, nx, ny, nz, btag,
                                                           cloud, Dx, Dy, Dz, lap, lapP);
    MGM_LAUNCHED();
}

// create_restriction_matrix / create_prolongation_matrix (mesh_functions.h:533-670)
__global__ void k_transfer_weights(int nt, const double *__restrict__ tx, const double *__restrict__ ty,
                                   const double *__restrict__ tz, const uint8_t *__restrict__ tbtag,
                                   const int *__restrict__ src_pt, int rows_from, int only_interior, int ks, int dim,
                                   int phs, MonoDev mono, const double *__restrict__ sxg, const double *__restrict__ syg,
                                   const double *__restrict__ szg, const int *__restrict__ scloud, double *W)
{
    extern __shared__ double sm[];
    const int m = ks, np = mono.np, N = m + np;
    double *aug = sm;
    double *sx = aug + (size_t)N * 2 * N, *sy = sx + m, *sz = sy + m;
    double *tmp = sz + m;  // [N]
    double *t = tmp + N;   // [N]
    int *perm = (int *)(t + N);
    const Team tm = Team::block();
    for (long i = blockIdx.x; i < nt; i += gridDim.x) {
        const bool skip = only_interior ? (tbtag[i] != 0) : (i < rows_from);
        if (skip) {
            for (int j = threadIdx.x; j < m; j += blockDim.x) W[i * ks + j] = 0.0;
            continue;
        }
        const int ip = src_pt[i];
        const int *cl = scloud + (long)ip * ks;
        stage_cloud(tm, cl, m, sxg, syg, szg, sx, sy, sz);
        tm.sync();
        build_aug(tm, m, np, dim, phs, mono, sx, sy, sz, aug, N);
        const double p1[3] = {tx[i], ty[i], tz[i]};
        const double seed[3] = {sxg[ip], syg[ip], szg[ip]};
        transfer_row(tm, m, np, dim, phs, mono, sx, sy, sz, p1, seed, tmp);
        tm.sync();
        gauss_jordan(tm, aug, perm, t, N);
        // multiply_vector_matrix_columnwise (mat_lib.h:720-726)
        for (int c = threadIdx.x; c < m; c += blockDim.x) W[i * ks + c] = row_times_inverse(tmp, aug, perm, N, c);
        __syncthreads();
    }
}

void transfer_weights(int nt, const double *tx, const double *ty, const double *tz, const uint8_t *tbtag,
                      const int *src_pt, int rows_from, int only_interior, int ks, int dim, int phs,
                      const Monomials &mono, const double *sx, const double *sy, const double *sz,
                      const int *scloud, double *W, cudaStream_t s)
{
    MGM_REQUIRE(ks >= 2 && ks <= kMaxK && ks + mono.np <= kMaxN, "transfer weights: stencil too large");
    if (nt <= 0) return;
    const int N = ks + mono.np;
    size_t smem = sizeof(double) * ((size_t)N * 2 * N + 3 * ks + 2 * N) + sizeof(int) * N;
    MGM_REQUIRE(smem <= 227 * 1024, "transfer weights: system does not fit in shared memory");
    MGM_CUDA(cudaFuncSetAttribute(k_transfer_weights, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_transfer_weights<<<weights_grid(nt), 128, smem, s>>>(nt, tx, ty, tz, tbtag, src_pt, rows_from, only_interior, ks,
                                                          dim, phs, to_dev(mono), sx, sy, sz, scloud, W);
    MGM_LAUNCHED();
}

// ===========================================================================
// layout helpers
// ===========================================================================
template <class T>
__global__ void k_transpose(const T *__restrict__ in, T *__restrict__ out, int rows, int cols)
{
    // in [rows][cols] -> out [cols][rows]
    __shared__ T tile[32][33];
    int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += 8) {
        int row = by + r, col = bx + threadIdx.x;
        if (row < rows && col < cols) tile[r][threadIdx.x] = in[(long)row * cols + col];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
        int col = bx + r, row = by + threadIdx.x;
        if (row < rows && col < cols) out[(long)col * rows + row] = tile[threadIdx.x][r];
    }
}

template <class T>
static void transpose(const T *in, T *out, int rows, int cols, cudaStream_t s)
{
    if (rows <= 0 || cols <= 0) return;
    dim3 grid(blocks_for(cols, 32), blocks_for(rows, 32)), block(32, 8);
    k_transpose<T><<<grid, block, 0, s>>>(in, out, rows, cols);
    MGM_LAUNCHED();
}

void transpose_rowmajor_to_ell_d(const double *in, double *out, int n, int k, cudaStream_t s) { transpose(in, out, n, k, s); }
void transpose_rowmajor_to_ell_i(const int *in, int *out, int n, int k, cudaStream_t s) { transpose(in, out, n, k, s); }
void transpose_ell_to_rowmajor_d(const double *in, double *out, int n, int k, cudaStream_t s) { transpose(in, out, k, n, s); }
void transpose_ell_to_rowmajor_i(const int *in, int *out, int n, int k, cudaStream_t s) { transpose(in, out, k, n, s); }

__global__ void k_d2f(const double *in, float *out, long n)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)in[i];
}
void convert_d2f(const double *in, float *out, long n, cudaStream_t s)
{
    if (n <= 0) return;
    k_d2f<<<blocks_for(n, 256), 256, 0, s>>>(in, out, n);
    MGM_LAUNCHED();
}

}  // namespace mgm
