// mpnn.cu -- learned warm start for the Poisson solve: a small message-passing
// network on the RBF-FD stencil graph, trained on the GPU by these kernels.
//
// Network (fixed shape): per node the inputs x_i = [b_i/rms(b), p_i/rms(p),
// dp_i/rms(dp), x_i, y_i, boundary tag] with dp = p_prev - p_prev2 the last
// pressure increment (0 when there is none); encoder h0 = relu(x W_e + c_e)
// (6 -> 64); four
// layers h' = relu([h_i | mean_j h_j | sum_j l_ij h_j] W_l + c_l) + h_i with
// j over the node's stencil and l_ij = h^2 lap_ij (192 -> 64); decoder
// y_i = h4_i . w_d + c_d.  Weights and activations are stored in BF16, every
// product is accumulated in FP32; the layer GEMM runs on the tensor cores
// (mma.sync m16n8k16 BF16 -> FP32) fused with the neighbour aggregation.
//
// The prediction is the shape of what the extrapolation misses,
// (p_new - p_prev) - dp.  The solve combines it with the extrapolation
// direction dp by the coefficients that minimise the FP64 residual, then runs
// the V-cycle-preconditioned FGMRES to the same tolerance as without it: the
// learned guess can only lower the starting residual, never replace the
// solver.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>

#include "ctx.cuh"

namespace mgm {

constexpr int kH = 64, kCat = 192, kFin = 6, kLayers = 4;
constexpr int kLayerParams = kCat * kH + kH;
constexpr int P_WE = 0, P_CE = kFin * kH, P_L0 = P_CE + kH;
constexpr int P_WD = P_L0 + kLayers * kLayerParams, P_CD = P_WD + kH;
constexpr int kNumParams = P_CD + 1;

typedef __nv_bfloat16 bf16;

struct MpnnState {
    int n = 0, k = 0;
    double d2 = 1;  // d_avg^2, scales lap weights to O(1)
    DBuf<float> params, grads, am, av;
    DBuf<bf16> WT[kLayers];  // [64][192]
    DBuf<bf16> WF[kLayers];  // the same in the forward GEMM's B-fragment order
    DBuf<float> lapS;        // row-major [n][k]
    DBuf<int> tptr, tpos;    // transpose adjacency: in-edges of node j as positions i*k+s, sorted
    DBuf<float> Arm;         // pinned Poisson operator, row-major [n][k] (FP32), for the residual loss
    float w_mse = 1.f, w_res = 0.f;
    DBuf<float> feat;        // [n][5]
    DBuf<bf16> h[kLayers + 1];
    DBuf<bf16> cat[kLayers];
    DBuf<float> z[kLayers + 1];
    DBuf<float> y, dy, dH, dHin, dz, dm;
    DBuf<double> scal;       // device scalars: [0..1] sum of squares of b, p; [2] loss; [5] of dp
    DBuf<float> ds;          // dataset: cap samples x kSlot x n (b_hat, p_hat, dp_hat, target)
    DBuf<double> dp;         // p_prev - p_prev2 of the sample being recorded
    int ds_cap = 0, ds_count = 0;
    int adam_t = 0;
    bool ready = false;
    const int *cloud = nullptr;  // level-0 cloud, row-major [n][k] (owned by the context)
};

// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 ld_bf2(const bf16 *p)
{
    const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162 *>(p);
    return __bfloat1622float2(v);
}
__device__ __forceinline__ void st_bf2(bf16 *p, float a, float b)
{
    *reinterpret_cast<__nv_bfloat162 *>(p) = __floats2bfloat162_rn(a, b);
}

template <int BS>
__device__ __forceinline__ double bsum_d(double v, double *sm)
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

// sum of squares of two vectors -> atomically into out[0], out[1] (zeroed before)
__global__ void k_sumsq2(int n, const double *a, const double *b, double *out)
{
    __shared__ double sm[32];
    double sa = 0, sb = 0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        sa += a[i] * a[i];
        sb += b[i] * b[i];
    }
    sa = bsum_d<256>(sa, sm);
    sb = bsum_d<256>(sb, sm);
    if (threadIdx.x == 0) { atomicAdd(out, sa); atomicAdd(out + 1, sb); }
}

__device__ __forceinline__ float inv_rms(double sumsq, int n)
{
    return sumsq > 0 ? (float)(1.0 / sqrt(sumsq / n)) : 0.f;
}

// dataset slot: b_hat, p_hat, dp_hat, target, each n floats
constexpr int kSlot = 4;

// inference features from the solver's b, p and last increment dp (double;
// dp may be null: no increment yet); ss: sums of squares of b, p, (dp)
__global__ void k_features(int n, const double *b, const double *p, const double *dp, const double *ss,
                           const double *x, const double *y, const uint8_t *btag, float *feat)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float sb = inv_rms(ss[0], n), sp = inv_rms(ss[1], n), sd = dp ? inv_rms(ss[5], n) : 0.f;
    float *f = feat + (long)i * kFin;
    f[0] = (float)b[i] * sb;
    f[1] = (float)p[i] * sp;
    f[2] = dp ? (float)dp[i] * sd : 0.f;
    f[3] = (float)x[i];
    f[4] = (float)y[i];
    f[5] = btag[i] ? 1.f : 0.f;
}

// training features from normalised dataset vectors
__global__ void k_features_ds(int n, const float *bh, const float *ph, const float *dh, const double *x,
                              const double *y, const uint8_t *btag, float *feat)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float *f = feat + (long)i * kFin;
    f[0] = bh[i];
    f[1] = ph[i];
    f[2] = dh[i];
    f[3] = (float)x[i];
    f[4] = (float)y[i];
    f[5] = btag[i] ? 1.f : 0.f;
}

// encoder: eight lanes per node (hidden features 8l..8l+7, one 16-byte store
// of h0), four nodes per warp, grid-stride over nodes; each lane keeps its 8
// columns of W_e and c_e in registers (loaded once), so the node loop reads
// only the 6 inputs.  Each feature's sum is c_e then the inputs in order.
__global__ void __launch_bounds__(256) k_encode(int n, const float *__restrict__ feat, const float *__restrict__ P,
                                                bf16 *__restrict__ h0, float *__restrict__ z0)
{
    const int c = 8 * (threadIdx.x & 7);
    float w[kFin][8], cb[8];
#pragma unroll
    for (int e = 0; e < 8; e++) cb[e] = __ldg(P + P_CE + c + e);
#pragma unroll
    for (int q = 0; q < kFin; q++)
#pragma unroll
        for (int e = 0; e < 8; e++) w[q][e] = __ldg(P + P_WE + q * kH + c + e);
    const long stride = (long)gridDim.x * (blockDim.x >> 3);
    for (long node = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 3; node < n; node += stride) {
        float f[kFin], a[8];
#pragma unroll
        for (int q = 0; q < kFin; q++) f[q] = __ldg(feat + node * kFin + q);
#pragma unroll
        for (int e = 0; e < 8; e++) a[e] = cb[e];
#pragma unroll
        for (int q = 0; q < kFin; q++)
#pragma unroll
            for (int e = 0; e < 8; e++) a[e] += f[q] * w[q][e];
        float r[8];
#pragma unroll
        for (int e = 0; e < 8; e++) r[e] = fmaxf(a[e], 0.f);
        uint4 u;
        __nv_bfloat162 *b = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
        for (int q = 0; q < 4; q++) b[q] = __floats2bfloat162_rn(r[2 * q], r[2 * q + 1]);
        *reinterpret_cast<uint4 *>(h0 + node * kH + c) = u;
        if (z0) {
            *reinterpret_cast<float4 *>(z0 + node * kH + c) = make_float4(a[0], a[1], a[2], a[3]);
            *reinterpret_cast<float4 *>(z0 + node * kH + c + 4) = make_float4(a[4], a[5], a[6], a[7]);
        }
    }
}

__device__ __forceinline__ void mma_bf16(float *c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

constexpr int kTile = 64, kPad = 200;  // rows per CTA, padded row length (bf16) of the smem tile

struct bf4 { __nv_bfloat162 a, b; };

// One message-passing layer for 64 nodes: gather [h_i | mean h_j | sum l_ij h_j]
// into shared memory (BF16), multiply by W (tensor cores, FP32 accumulate),
// bias + relu + residual, store h' (BF16); in training also z and the row.
// Aggregation: eight lanes per node (8 features, one 16-byte load per lane
// and neighbour row), four nodes per warp at a time; each lane holds the
// node's stencil slots l, l+8, ... and the group shares them by shuffles;
// the neighbour rows of kGather slots are in flight at once.  Each feature's
// sums run over the slots in order.  W (24 KB) is read through L1.  Six slots
// in flight at 80 registers (6 CTAs, 24 warps per SM) measured 9% faster per
// layer than ten at 128 registers (4 CTAs); the bits are the same.
constexpr int kGather = 6;

__device__ __forceinline__ void unpack8(const uint4 &u, float *f)
{
    const __nv_bfloat162 *b = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const float2 v = __bfloat1622float2(b[q]);
        f[2 * q] = v.x;
        f[2 * q + 1] = v.y;
    }
}
__device__ __forceinline__ uint4 pack8(const float *f)
{
    uint4 u;
    __nv_bfloat162 *b = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
    for (int q = 0; q < 4; q++) b[q] = __floats2bfloat162_rn(f[2 * q], f[2 * q + 1]);
    return u;
}

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3)
{
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}

// W^T in the order of the mma.sync B fragments: for k-step ks (16 of the 192
// inputs), n-tile pair p (16 of the 64 outputs) and lane l, one 16-byte word
// {b0, b1 of n-tile 2p, b0, b1 of n-tile 2p + 1}; a warp reads a pair's
// fragments as 512 contiguous bytes (kept in L1 for every CTA of the SM)
__host__ __device__ constexpr int frag_pos(int f, int c)
{
    // f: output (n) 0..63, c: input (k) 0..191 -> position in the fragment-ordered copy (bf16 units)
    return (((c / 16) * 4 + (f / 16)) * 32 + (f % 8) * 4 + (c % 8) / 2) * 8 + (((f / 8) % 2) * 2 + (c % 16) / 8) * 2 +
           (c % 2);
}

__global__ void __launch_bounds__(128, 6) k_mp_layer(int n, int k, const int *__restrict__ cloud,
                                                  const float *__restrict__ lapS, float inv_k,
                                                  const bf16 *__restrict__ h_in, const bf16 *__restrict__ WF,
                                                  const float *__restrict__ bias, bf16 *__restrict__ h_out,
                                                  float *__restrict__ z_out, bf16 *__restrict__ cat_out,
                                                  const float *__restrict__ dec, float *__restrict__ y_out)
{
    __shared__ __align__(16) bf16 Xs[kTile][kPad];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int grp = lane >> 3, gl = lane & 7;
    const unsigned full = 0xffffffffu;  // rows past n are clamped, so all lanes stay converged
    const long base = (long)blockIdx.x * kTile;
    for (int rr = 0; rr < kTile / 16; rr++) {
        const int row = warp * 16 + rr * 4 + grp;
        const bool valid = base + row < n;
        const long i = valid ? base + row : (long)n - 1;
        float sf[8], mn[8], lp[8];
#pragma unroll
        for (int e = 0; e < 8; e++) mn[e] = lp[e] = 0.f;
        unpack8(__ldg(reinterpret_cast<const uint4 *>(h_in + i * kH + 8 * gl)), sf);
        // the node's slots gl, gl + 8, ... (k <= 64)
        int cl[8];
        float wl[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int j = gl + 8 * e;
            cl[e] = j < k ? __ldg(cloud + i * k + j) : 0;
            wl[e] = j < k ? __ldg(lapS + i * k + j) : 0.f;
        }
#pragma unroll
        for (int j0 = 0; j0 < 64; j0 += kGather) {
            if (j0 >= k) break;
            uint4 v[kGather];
            float wj[kGather];
#pragma unroll
            for (int e = 0; e < kGather; e++) {
                const int j = j0 + e;
                if (j >= 64) { wj[e] = 0.f; v[e] = make_uint4(0, 0, 0, 0); continue; }
                const int cs = __shfl_sync(full, cl[j >> 3], j & 7, 8);
                wj[e] = __shfl_sync(full, wl[j >> 3], j & 7, 8);
                v[e] = j < k ? __ldg(reinterpret_cast<const uint4 *>(h_in + (long)cs * kH + 8 * gl))
                             : make_uint4(0, 0, 0, 0);
            }
#pragma unroll
            for (int e = 0; e < kGather; e++) {
                if (j0 + e >= k) break;
                float f[8];
                unpack8(v[e], f);
#pragma unroll
                for (int c = 0; c < 8; c++) {
                    mn[c] += f[c];
                    lp[c] += wj[e] * f[c];
                }
            }
        }
#pragma unroll
        for (int e = 0; e < 8; e++) {
            mn[e] *= inv_k;
            if (!valid) sf[e] = mn[e] = lp[e] = 0.f;
        }
        *reinterpret_cast<uint4 *>(&Xs[row][8 * gl]) = pack8(sf);
        *reinterpret_cast<uint4 *>(&Xs[row][kH + 8 * gl]) = pack8(mn);
        *reinterpret_cast<uint4 *>(&Xs[row][2 * kH + 8 * gl]) = pack8(lp);
    }
    __syncthreads();
    const int g = lane >> 2, t = lane & 3, r0 = warp * 16;
    // A fragments by ldmatrix: lanes 8q..8q+7 address rows r0 + (q & 1) * 8 + 0..7 at column (q >> 1) * 8
    const int q = lane >> 3, rq = lane & 7;
    const uint32_t a_addr = (uint32_t)__cvta_generic_to_shared(&Xs[r0 + rq + 8 * (q & 1)][8 * (q >> 1)]);
    const uint4 *Wq = reinterpret_cast<const uint4 *>(WF) + lane;
    float acc[8][4];
#pragma unroll
    for (int e = 0; e < 8; e++) acc[e][0] = acc[e][1] = acc[e][2] = acc[e][3] = 0.f;
#pragma unroll
    for (int ks = 0; ks < kCat / 16; ks++) {
        uint32_t a0, a1, a2, a3;
        ldsm_x4(a_addr + ks * 16 * (uint32_t)sizeof(bf16), a0, a1, a2, a3);
#pragma unroll
        for (int p = 0; p < 4; p++) {
            const uint4 b = __ldg(Wq + (ks * 4 + p) * 32);
            mma_bf16(acc[2 * p], a0, a1, a2, a3, b.x, b.y);
            mma_bf16(acc[2 * p + 1], a0, a1, a2, a3, b.z, b.w);
        }
    }
    float yp[2] = {0.f, 0.f};
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
        const int col = nt * 8 + 2 * t;
#pragma unroll
        for (int hh = 0; hh < 2; hh++) {
            const int row = r0 + g + 8 * hh;
            const long i = base + row;
            if (i >= n) continue;
            const float z0 = acc[nt][2 * hh] + bias[col], z1 = acc[nt][2 * hh + 1] + bias[col + 1];
            const float2 res = ld_bf2(&Xs[row][col]);
            const __nv_bfloat162 o = __floats2bfloat162_rn(fmaxf(z0, 0.f) + res.x, fmaxf(z1, 0.f) + res.y);
            if (h_out) *reinterpret_cast<__nv_bfloat162 *>(h_out + i * kH + col) = o;
            if (z_out) { z_out[i * kH + col] = z0; z_out[i * kH + col + 1] = z1; }
            if (y_out) {
                const float2 of = __bfloat1622float2(o);
                yp[hh] += of.x * __ldg(dec + P_WD + col) + of.y * __ldg(dec + P_WD + col + 1);
            }
        }
    }
    if (y_out) {
        // decoder: the four lanes of a row hold its 64 features in 16-column
        // parts; the row's output is their sum plus c_d
#pragma unroll
        for (int hh = 0; hh < 2; hh++) {
            float v = yp[hh];
            v += __shfl_xor_sync(0xffffffffu, v, 1);
            v += __shfl_xor_sync(0xffffffffu, v, 2);
            const long i = base + r0 + g + 8 * hh;
            if (t == 0 && i < n) y_out[i] = v + __ldg(dec + P_CD);
        }
    }
    if (cat_out) {
        for (int w = tid; w < kTile * (kCat / 2); w += blockDim.x) {
            const int r = w / (kCat / 2), cw = w % (kCat / 2);
            if (base + r < n)
                reinterpret_cast<uint32_t *>(cat_out + (base + r) * kCat)[cw] =
                    reinterpret_cast<const uint32_t *>(&Xs[r][0])[cw];
        }
    }
}

// decoder: warp per node
__global__ void __launch_bounds__(256) k_decode(int n, const bf16 *h, const float *P, float *y)
{
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= n) return;
    const float2 v = ld_bf2(h + (long)w * kH + 2 * lane);
    float s = v.x * P[P_WD + 2 * lane] + v.y * P[P_WD + 2 * lane + 1];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) y[w] = s + P[P_CD];
}

// ---------------------------------------------------------------------------
// backward
// ---------------------------------------------------------------------------
// loss = mean (y - t)^2 ; dy = 2 (y - t) / n ; loss accumulated into *loss
__global__ void k_loss(int n, const float *y, const float *t, float *dy, double *loss)
{
    __shared__ double sm[32];
    double s = 0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float r = y[i] - t[i];
        dy[i] = 2.f * r / n;
        s += (double)r * r;
    }
    s = bsum_d<256>(s, sm);
    if (threadIdx.x == 0) atomicAdd(loss, s / n);
}

// dH4 = dy w_d ; grads of w_d, c_d (warp per node, grid-stride, one atomic per lane at the end)
__global__ void __launch_bounds__(256) k_decode_bwd(int n, const bf16 *h, const float *dy, const float *P, float *dH,
                                                    float *G)
{
    const int lane = threadIdx.x & 31;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    float gw0 = 0, gw1 = 0, gc = 0;
    const float w0 = P[P_WD + 2 * lane], w1 = P[P_WD + 2 * lane + 1];
    for (long i = (((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < n; i += nw) {
        const float d = dy[i];
        const float2 v = ld_bf2(h + i * kH + 2 * lane);
        gw0 += v.x * d; gw1 += v.y * d;
        gc += d;
        dH[i * kH + 2 * lane] = d * w0;
        dH[i * kH + 2 * lane + 1] = d * w1;
    }
    atomicAdd(&G[P_WD + 2 * lane], gw0);
    atomicAdd(&G[P_WD + 2 * lane + 1], gw1);
    if (lane == 0) atomicAdd(&G[P_CD], gc);
}

// dz = dH * [z > 0] ; dHin = dH (residual path) ; bias grads
__global__ void __launch_bounds__(256) k_relu_bwd(int n, const float *dH, const float *z, float *dz, float *dHin,
                                                  float *gbias)
{
    const int lane = threadIdx.x & 31;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    float g0 = 0, g1 = 0;
    for (long i = (((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < n; i += nw) {
        const long o = i * kH + 2 * lane;
        const float d0 = z[o] > 0.f ? dH[o] : 0.f, d1 = z[o + 1] > 0.f ? dH[o + 1] : 0.f;
        dz[o] = d0; dz[o + 1] = d1;
        if (dHin) { dHin[o] = dH[o]; dHin[o + 1] = dH[o + 1]; }
        g0 += d0; g1 += d1;
    }
    atomicAdd(&gbias[2 * lane], g0);
    atomicAdd(&gbias[2 * lane + 1], g1);
}

// gW[kk][f] += sum_i cat[i][kk] dz[i][f]  (thread kk, 64 accumulators; node chunks per CTA)
__global__ void __launch_bounds__(192) k_dW(int n, int chunk, const bf16 *cat, const float *dz, float *gW)
{
    __shared__ float dzs[16][kH];
    const int kk = threadIdx.x;
    const long i0 = (long)blockIdx.x * chunk, i1 = min((long)n, i0 + chunk);
    float acc[kH];
#pragma unroll
    for (int f = 0; f < kH; f++) acc[f] = 0.f;
    for (long ib = i0; ib < i1; ib += 16) {
        __syncthreads();
        for (int e = threadIdx.x; e < 16 * kH; e += blockDim.x) {
            const long i = ib + e / kH;
            dzs[e / kH][e % kH] = i < i1 ? dz[i * kH + e % kH] : 0.f;
        }
        __syncthreads();
        const int m = (int)min(16L, i1 - ib);
        for (int q = 0; q < m; q++) {
            const float a = __bfloat162float(cat[(ib + q) * kCat + kk]);
#pragma unroll
            for (int f = 0; f < kH; f++) acc[f] += a * dzs[q][f];
        }
    }
#pragma unroll
    for (int f = 0; f < kH; f++) atomicAdd(&gW[kk * kH + f], acc[f]);
}

// dcat = dz W^T: self part added to dHin, mean/lap parts into dm [n][128]
__global__ void __launch_bounds__(192) k_dcat(int n, const float *dz, const bf16 *WT, float *dHin, float *dm)
{
    __shared__ bf16 Wsh[kCat][kH + 2];
    __shared__ float dzs[16][kH];
    const int kk = threadIdx.x;
    for (int e = threadIdx.x; e < kCat * kH; e += blockDim.x) {
        const int f = e / kCat, c = e % kCat;  // WT is [64][192]
        Wsh[c][f] = WT[e];
    }
    for (long ib = (long)blockIdx.x * 16; ib < n; ib += (long)gridDim.x * 16) {
        __syncthreads();
        for (int e = threadIdx.x; e < 16 * kH; e += blockDim.x) {
            const long i = ib + e / kH;
            dzs[e / kH][e % kH] = i < n ? dz[i * kH + e % kH] : 0.f;
        }
        __syncthreads();
        for (int q = 0; q < 16; q++) {
            const long i = ib + q;
            if (i >= n) break;
            float s = 0.f;
#pragma unroll 16
            for (int f = 0; f < kH; f++) s += dzs[q][f] * __bfloat162float(Wsh[kk][f]);
            if (kk < kH) dHin[i * kH + kk] += s;
            else dm[i * 128 + (kk - kH)] = s;
        }
    }
}

// dHin[j] += sum over in-edges (i, l_ij): dm_mean[i] / k + l_ij dm_lap[i]
__global__ void __launch_bounds__(256) k_scatter_T(int n, int k, float inv_k, const int *tptr, const int *tpos,
                                                   const float *lapS, const float *dm, float *dHin)
{
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (j >= n) return;
    float a0 = 0, a1 = 0;
    for (int e = tptr[j]; e < tptr[j + 1]; e++) {
        const int pos = tpos[e];
        const long i = pos / k;
        const float w = lapS[pos];
        const float *r = dm + i * 128;
        a0 += inv_k * r[2 * lane] + w * r[kH + 2 * lane];
        a1 += inv_k * r[2 * lane + 1] + w * r[kH + 2 * lane + 1];
    }
    dHin[(long)j * kH + 2 * lane] += a0;
    dHin[(long)j * kH + 2 * lane + 1] += a1;
}

// encoder grads
__global__ void __launch_bounds__(256) k_encode_bwd(int n, const float *feat, const float *z0, const float *dH,
                                                    float *G)
{
    const int lane = threadIdx.x & 31;
    const long nw = ((long)gridDim.x * blockDim.x) >> 5;
    float gw[kFin][2] = {}, gc0 = 0, gc1 = 0;
    for (long i = (((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < n; i += nw) {
        const long o = i * kH + 2 * lane;
        const float d0 = z0[o] > 0.f ? dH[o] : 0.f, d1 = z0[o + 1] > 0.f ? dH[o + 1] : 0.f;
#pragma unroll
        for (int q = 0; q < kFin; q++) {
            const float xv = feat[i * kFin + q];
            gw[q][0] += xv * d0;
            gw[q][1] += xv * d1;
        }
        gc0 += d0; gc1 += d1;
    }
#pragma unroll
    for (int q = 0; q < kFin; q++) {
        atomicAdd(&G[P_WE + q * kH + 2 * lane], gw[q][0]);
        atomicAdd(&G[P_WE + q * kH + 2 * lane + 1], gw[q][1]);
    }
    atomicAdd(&G[P_CE + 2 * lane], gc0);
    atomicAdd(&G[P_CE + 2 * lane + 1], gc1);
}

__global__ void k_adam(int np, float *P, const float *G, float *m, float *v, float lr, float b1, float b2, float eps,
                       float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const float g = G[i];
    const float mi = b1 * m[i] + (1 - b1) * g, vi = b2 * v[i] + (1 - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// BF16 copies of the layer weights: transposed to [64][192] (the backward
// pass) and in the forward GEMM's B-fragment order (frag_pos)
__global__ void k_refresh_WT(const float *P, bf16 *W0, bf16 *W1, bf16 *W2, bf16 *W3, bf16 *F0, bf16 *F1, bf16 *F2,
                             bf16 *F3)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= kLayers * kH * kCat) return;
    const int l = e / (kH * kCat), r = e % (kH * kCat), f = r / kCat, c = r % kCat;
    bf16 *dst[4] = {W0, W1, W2, W3}, *frg[4] = {F0, F1, F2, F3};
    const bf16 w = __float2bfloat16(P[P_L0 + l * kLayerParams + c * kH + f]);
    dst[l][f * kCat + c] = w;
    frg[l][frag_pos(f, c)] = w;
}

// scaled lap weights row-major from the ELL operator
__global__ void k_lapS(int n, int k, const double *lap, double d2, float *out)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)n * k) return;
    const int i = (int)(t / k), j = (int)(t % k);
    out[t] = (float)(lap[(long)j * n + i] * d2);
}

__global__ void k_count_in(int n, int k, const int *cloud, int *deg)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < (long)n * k) atomicAdd(&deg[cloud[t]], 1);
}

__global__ void k_fill_in(int n, int k, const int *cloud, int *fill, int *tpos)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)n * k) return;
    const int pos = atomicAdd(&fill[cloud[t]], 1);
    tpos[pos] = (int)t;
}

// deterministic order of each node's in-edges: by position i*k+s
__global__ void k_sort_in(int n, const int *tptr, int *tpos)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    for (int a = tptr[j] + 1; a < tptr[j + 1]; a++) {
        const int v = tpos[a];
        int b = a;
        while (b > tptr[j] && tpos[b - 1] > v) { tpos[b] = tpos[b - 1]; b--; }
        tpos[b] = v;
    }
}

// row-major FP32 copy of an ELL FP64 operator
__global__ void k_rowmajor_f(int n, int k, const double *A, float *out)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)n * k) return;
    const int i = (int)(t / k), j = (int)(t % k);
    out[t] = (float)A[(long)j * n + i];
}

// residual loss, forward: r = A (t - y), q = A t ; sums of squares -> acc[0], acc[1]
__global__ void k_res_fwd(int n, int k, const int *cloud, const float *Arm, const float *t, const float *y, float *r,
                          double *acc)
{
    __shared__ double sm[32];
    double sr = 0, sq = 0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        float a = 0.f, b = 0.f;
        for (int s = 0; s < k; s++) {
            const long o = i * k + s;
            const int c = cloud[o];
            a += Arm[o] * (t[c] - y[c]);
            b += Arm[o] * t[c];
        }
        r[i] = a;
        sr += (double)a * a;
        sq += (double)b * b;
    }
    sr = bsum_d<256>(sr, sm);
    sq = bsum_d<256>(sq, sm);
    if (threadIdx.x == 0) { atomicAdd(acc, sr); atomicAdd(acc + 1, sq); }
}

// dy = w_res * (-2 A^T r / |A t|^2) + w_mse * 2 (y - t) / n ; loss += w_res |r|^2/|A t|^2 (mse part added by k_loss)
__global__ void k_res_bwd(int n, int k, const int *tptr, const int *tpos, const float *Arm, const float *r,
                          const double *acc, float w_res, float *dy)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double Q = acc[1] > 0 ? acc[1] : 1.0;
    float s = 0.f;
    for (int e = tptr[j]; e < tptr[j + 1]; e++) {
        const int pos = tpos[e];
        s += Arm[pos] * r[pos / k];
    }
    dy[j] += (float)(w_res * (-2.0 * s / Q));
}

// dataset record: slot <- (b/rms b, p_prev/rms, dp/rms, target/rms) with
// dp = p_prev - p_prev2 and target = (p_new - p_prev) - dp, the part of the
// new increment the extrapolation misses (p_new - p_prev when there is no
// p_prev2: pprev2 null, dp_hat = 0); ss[0..1] sums of squares of b, p_prev,
// ss[2] of the target, ss[5] of dp
__global__ void k_record(int n, const double *b, const double *pprev, const double *pprev2, const double *pnew,
                         const double *ss, float *slot)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float sb = inv_rms(ss[0], n), sp = inv_rms(ss[1], n), sd = inv_rms(ss[2], n);
    const float sq = pprev2 ? inv_rms(ss[5], n) : 0.f;
    const double dp = pprev2 ? pprev[i] - pprev2[i] : 0.0;
    slot[i] = (float)b[i] * sb;
    slot[n + i] = (float)pprev[i] * sp;
    slot[2 * n + i] = (float)dp * sq;
    slot[3 * n + i] = (float)((pnew[i] - pprev[i]) - dp) * sd;
}

// sum of (a - b - c)^2 (c may be null) -> atomically into out[0]
__global__ void k_sumsq_diff2(int n, const double *a, const double *b, const double *c, double *out)
{
    __shared__ double sm[32];
    double s = 0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double d = a[i] - b[i] - (c ? c[i] : 0.0);
        s += d * d;
    }
    s = bsum_d<256>(s, sm);
    if (threadIdx.x == 0) atomicAdd(out, s);
}

__global__ void k_diff(int n, const double *a, const double *b, double *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[i] - b[i];
}

__global__ void k_sumsq_diff(int n, const double *a, const double *b, double *out)
{
    __shared__ double sm[32];
    double s = 0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double d = a[i] - b[i];
        s += d * d;
    }
    s = bsum_d<256>(s, sm);
    if (threadIdx.x == 0) atomicAdd(out, s);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static int red_blocks(int n) { return std::max(1, std::min(blocks_for(n, 256), 148 * 4)); }
static int warp_blocks(long n) { return blocks_for(n * 32, 256); }

static void refresh_weights(MpnnState &M, cudaStream_t s)
{
    k_refresh_WT<<<blocks_for(kLayers * kH * kCat, 256), 256, 0, s>>>(M.params.p, M.WT[0].p, M.WT[1].p, M.WT[2].p,
                                                                      M.WT[3].p, M.WF[0].p, M.WF[1].p, M.WF[2].p,
                                                                      M.WF[3].p);
    MGM_LAUNCHED();
}

// forward from M.feat; train = keep z / cat for the backward pass; output M.y
static void forward(MpnnState &M, bool train, cudaStream_t s)
{
    const int n = M.n;
    const float *P = M.params.p;
    k_encode<<<std::min(blocks_for((long)n * 8, 256), 148 * 8), 256, 0, s>>>(n, M.feat.p, P, M.h[0].p,
                                                                             train ? M.z[0].p : nullptr);
    MGM_LAUNCHED();
    for (int l = 0; l < kLayers; l++) {
        // inference: the last layer decodes in its epilogue and stores no h4
        const bool dec = !train && l == kLayers - 1;
        k_mp_layer<<<blocks_for(n, kTile), 128, 0, s>>>(n, M.k, M.cloud, M.lapS.p, 1.f / M.k, M.h[l].p, M.WF[l].p,
                                                       P + P_L0 + l * kLayerParams + kCat * kH,
                                                       dec ? nullptr : M.h[l + 1].p, train ? M.z[l + 1].p : nullptr,
                                                       train ? M.cat[l].p : nullptr, dec ? P : nullptr,
                                                       dec ? M.y.p : nullptr);
        MGM_LAUNCHED();
    }
    if (train) {
        k_decode<<<warp_blocks(n), 256, 0, s>>>(n, M.h[kLayers].p, P, M.y.p);
        MGM_LAUNCHED();
    }
}

// loss w_mse * mean (y - t)^2 + w_res * |A (t - y)|^2 / |A t|^2 and dL/dy; loss -> M.scal[2]
__global__ void k_scale_mse(int n, float w, float *dy)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dy[i] *= w;
}
__global__ void k_add_loss(const double *acc, double w_mse, double w_res, double *loss)
{
    const double Q = acc[1] > 0 ? acc[1] : 1.0;
    *loss = w_mse * (*loss) + w_res * acc[0] / Q;
}

static void loss_head(MpnnState &M, const float *t, cudaStream_t s)
{
    const int n = M.n;
    MGM_CUDA(cudaMemsetAsync(M.scal.p + 2, 0, 3 * sizeof(double), s));
    k_loss<<<red_blocks(n), 256, 0, s>>>(n, M.y.p, t, M.dy.p, M.scal.p + 2);
    MGM_LAUNCHED();
    k_scale_mse<<<blocks_for(n, 256), 256, 0, s>>>(n, M.w_mse, M.dy.p);
    MGM_LAUNCHED();
    if (M.w_res > 0.f) {
        k_res_fwd<<<red_blocks(n), 256, 0, s>>>(n, M.k, M.cloud, M.Arm.p, t, M.y.p, M.dz.p, M.scal.p + 3);
        MGM_LAUNCHED();
        k_res_bwd<<<blocks_for(n, 256), 256, 0, s>>>(n, M.k, M.tptr.p, M.tpos.p, M.Arm.p, M.dz.p, M.scal.p + 3,
                                                    M.w_res, M.dy.p);
        MGM_LAUNCHED();
    }
    k_add_loss<<<1, 1, 0, s>>>(M.scal.p + 3, M.w_mse, M.w_res, M.scal.p + 2);
    MGM_LAUNCHED();
}

// loss against target t and the full gradient into M.grads (zeroed here); loss -> M.scal[2]
static void loss_and_grad(MpnnState &M, const float *t, cudaStream_t s)
{
    const int n = M.n;
    MGM_CUDA(cudaMemsetAsync(M.grads.p, 0, sizeof(float) * kNumParams, s));
    forward(M, true, s);
    loss_head(M, t, s);
    float *G = M.grads.p;
    k_decode_bwd<<<red_blocks(n), 256, 0, s>>>(n, M.h[kLayers].p, M.dy.p, M.params.p, M.dH.p, G);
    MGM_LAUNCHED();
    const int chunk = std::max(64, blocks_for(n, 148 * 4));
    for (int l = kLayers - 1; l >= 0; l--) {
        float *gl = G + P_L0 + l * kLayerParams;
        k_relu_bwd<<<red_blocks(n), 256, 0, s>>>(n, M.dH.p, M.z[l + 1].p, M.dz.p, M.dHin.p, gl + kCat * kH);
        MGM_LAUNCHED();
        k_dW<<<blocks_for(n, chunk), 192, 0, s>>>(n, chunk, M.cat[l].p, M.dz.p, gl);
        MGM_LAUNCHED();
        k_dcat<<<std::min(blocks_for(n, 16), 148 * 8), 192, 0, s>>>(n, M.dz.p, M.WT[l].p, M.dHin.p, M.dm.p);
        MGM_LAUNCHED();
        k_scatter_T<<<warp_blocks(n), 256, 0, s>>>(n, M.k, 1.f / M.k, M.tptr.p, M.tpos.p, M.lapS.p, M.dm.p, M.dHin.p);
        MGM_LAUNCHED();
        std::swap(M.dH.p, M.dHin.p);
    }
    k_encode_bwd<<<red_blocks(n), 256, 0, s>>>(n, M.feat.p, M.z[0].p, M.dH.p, G);
    MGM_LAUNCHED();
}

static void adam_step(MpnnState &M, float lr, cudaStream_t s)
{
    M.adam_t++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)M.adam_t), c2 = 1.f - powf(b2, (float)M.adam_t);
    k_adam<<<blocks_for(kNumParams, 256), 256, 0, s>>>(kNumParams, M.params.p, M.grads.p, M.am.p, M.av.p, lr, b1, b2,
                                                      1e-8f, c1, c2);
    MGM_LAUNCHED();
    refresh_weights(M, s);
}

// deterministic pseudo-random initial weights (He-scaled uniform), host-generated
static void init_params(std::vector<float> &P, unsigned long long seed)
{
    P.assign(kNumParams, 0.f);
    unsigned long long x = seed * 0x9E3779B97F4A7C15ULL + 1;
    auto rnd = [&]() {
        x ^= x << 13; x ^= x >> 7; x ^= x << 17;
        return (float)((x >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
    };
    const float se = sqrtf(6.f / kFin), sl = sqrtf(6.f / kCat) * 0.5f, sd = sqrtf(6.f / kH) * 0.5f;
    for (int i = 0; i < kFin * kH; i++) P[P_WE + i] = se * rnd();
    for (int l = 0; l < kLayers; l++)
        for (int i = 0; i < kCat * kH; i++) P[P_L0 + l * kLayerParams + i] = sl * rnd();
    for (int i = 0; i < kH; i++) P[P_WD + i] = sd * rnd();
}

MpnnState &state(mgm_ctx *c)
{
    MGM_REQUIRE(c->mpnn && c->mpnn->ready, "learned warm start not initialised (mgm_mpnn_init)");
    return *c->mpnn;
}

// The learned direction for the current Poisson system: b, p and the last
// pressure increment dp (device; dp all zero when there is none) -> out
// (device, precision T).  Called by the FGMRES of mgm_api.cu.
template <class T>
__global__ void k_to_T(int n, const float *y, T *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (T)y[i];
}

bool warm_start_enabled(mgm_ctx *c)
{
    return c->mpnn && c->mpnn->ready && (c->guess_flags & MGM_GUESS_LEARNED) && !c->warm_suspended;
}

template <class T>
void warm_direction(mgm_ctx *c, const double *b, const double *p, const double *dp, T *out, cudaStream_t s)
{
    MpnnState &M = *c->mpnn;
    Level &L = c->L[0];
    MGM_CUDA(cudaMemsetAsync(M.scal.p, 0, 6 * sizeof(double), s));
    k_sumsq2<<<red_blocks(M.n), 256, 0, s>>>(M.n, b, p, M.scal.p);
    MGM_LAUNCHED();
    k_sumsq2<<<red_blocks(M.n), 256, 0, s>>>(M.n, dp, dp, M.scal.p + 4);  // [5] = |dp|^2
    MGM_LAUNCHED();
    k_features<<<blocks_for(M.n, 256), 256, 0, s>>>(M.n, b, p, dp, M.scal.p, L.x.p, L.y.p, L.btag.p, M.feat.p);
    MGM_LAUNCHED();
    forward(M, false, s);
    k_to_T<T><<<blocks_for(M.n, 256), 256, 0, s>>>(M.n, M.y.p, out);
    MGM_LAUNCHED();
}
template void warm_direction<double>(mgm_ctx *, const double *, const double *, const double *, double *,
                                     cudaStream_t);
template void warm_direction<float>(mgm_ctx *, const double *, const double *, const double *, float *,
                                    cudaStream_t);

// record one sample (b, p_prev, p_prev - p_prev2, p_new - p_prev) into the
// dataset ring (pprev2 null: no earlier pressure)
void record_sample(mgm_ctx *c, const double *b, const double *pprev, const double *pprev2, const double *pnew,
                   cudaStream_t s)
{
    MpnnState &M = *c->mpnn;
    if (M.ds_cap == 0) return;
    const int slot = M.ds_count % M.ds_cap;
    MGM_CUDA(cudaMemsetAsync(M.scal.p, 0, 6 * sizeof(double), s));
    k_sumsq2<<<red_blocks(M.n), 256, 0, s>>>(M.n, b, pprev, M.scal.p);
    MGM_LAUNCHED();
    if (pprev2) {
        k_sumsq_diff<<<red_blocks(M.n), 256, 0, s>>>(M.n, pprev, pprev2, M.scal.p + 5);
        MGM_LAUNCHED();
        k_diff<<<blocks_for(M.n, 256), 256, 0, s>>>(M.n, pprev, pprev2, M.dp.p);
        MGM_LAUNCHED();
    }
    k_sumsq_diff2<<<red_blocks(M.n), 256, 0, s>>>(M.n, pnew, pprev, pprev2 ? M.dp.p : nullptr, M.scal.p + 2);
    MGM_LAUNCHED();
    k_record<<<blocks_for(M.n, 256), 256, 0, s>>>(M.n, b, pprev, pprev2, pnew, M.scal.p,
                                                  M.ds.p + (size_t)slot * kSlot * M.n);
    MGM_LAUNCHED();
    M.ds_count++;
}

void destroy_mpnn(mgm_ctx *c)
{
    delete c->mpnn;
    c->mpnn = nullptr;
}

}  // namespace mgm

using namespace mgm;

extern "C" {

int mgm_mpnn_init(mgm_ctx *c, unsigned long long seed, int dataset_capacity)
{
    try {
        MGM_REQUIRE(c && c->setup_done, "mgm_mpnn_init: call mgm_setup first");
        MGM_REQUIRE(dataset_capacity >= 0, "mgm_mpnn_init: negative capacity");
        MGM_CUDA(cudaSetDevice(c->device));
        cudaStream_t s = c->s;
        Level &L = c->L[0];
        MGM_REQUIRE(L.k <= 64, "mgm_mpnn_init: stencils wider than 64 are not supported by the network");
        delete c->mpnn;
        c->mpnn = new MpnnState();
        MpnnState &M = *c->mpnn;
        M.n = L.n; M.k = L.k; M.d2 = L.d_avg * L.d_avg; M.cloud = L.cloud.p;
        const size_t n = L.n, nk = (size_t)L.n * L.k;
        M.params.alloc(kNumParams); M.grads.alloc(kNumParams); M.am.alloc(kNumParams); M.av.alloc(kNumParams);
        M.am.zero(s); M.av.zero(s);
        std::vector<float> hp;
        init_params(hp, seed);
        M.params.upload(hp.data(), kNumParams, s);
        for (auto &w : M.WT) w.alloc((size_t)kH * kCat);
        for (auto &w : M.WF) w.alloc((size_t)kH * kCat);
        M.lapS.alloc(nk);
        k_lapS<<<blocks_for((long)nk, 256), 256, 0, s>>>(L.n, L.k, L.lap.p, M.d2, M.lapS.p);
        MGM_LAUNCHED();
        // transpose adjacency for the backward gather
        DBuf<int> deg(n), fill(n);
        deg.zero(s);
        M.tptr.alloc(n + 1);
        M.tpos.alloc(nk);
        M.Arm.alloc(nk);
        k_rowmajor_f<<<blocks_for((long)nk, 256), 256, 0, s>>>(L.n, L.k, L.A64.p, M.Arm.p);
        MGM_LAUNCHED();
        k_count_in<<<blocks_for((long)nk, 256), 256, 0, s>>>(L.n, L.k, L.cloud.p, deg.p);
        MGM_LAUNCHED();
        scan_exclusive(deg.p, M.tptr.p, L.n, M.tptr.p + n, s);
        MGM_CUDA(cudaMemcpyAsync(fill.p, M.tptr.p, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
        k_fill_in<<<blocks_for((long)nk, 256), 256, 0, s>>>(L.n, L.k, L.cloud.p, fill.p, M.tpos.p);
        MGM_LAUNCHED();
        k_sort_in<<<blocks_for(L.n, 256), 256, 0, s>>>(L.n, M.tptr.p, M.tpos.p);
        MGM_LAUNCHED();
        M.feat.alloc(n * kFin);
        for (auto &h : M.h) h.alloc(n * kH);
        for (auto &ct : M.cat) ct.alloc(n * kCat);
        for (auto &z : M.z) z.alloc(n * kH);
        M.y.alloc(n); M.dy.alloc(n); M.dH.alloc(n * kH); M.dHin.alloc(n * kH); M.dz.alloc(n * kH);
        M.dm.alloc(n * 128);
        M.scal.alloc(8);
        M.dp.alloc(n);
        M.ds_cap = dataset_capacity;
        M.ds_count = 0;
        if (dataset_capacity > 0) M.ds.alloc((size_t)dataset_capacity * kSlot * n);
        refresh_weights(M, s);
        MGM_CUDA(cudaStreamSynchronize(s));
        M.ready = true;
        return MGM_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    }
}

int mgm_mpnn_num_params(void) { return kNumParams; }

int mgm_mpnn_params(mgm_ctx *c, float *get, const float *set)
{
    try {
        MpnnState &M = state(c);
        cudaStream_t s = c->s;
        if (set) {
            M.params.upload(set, kNumParams, s);
            refresh_weights(M, s);
        }
        if (get) M.params.download(get, kNumParams, s);
        MGM_CUDA(cudaStreamSynchronize(s));
        return MGM_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    }
}

// loss and gradient for one sample given normalised host vectors (b_hat, p_hat, dp_hat, target)
int mgm_mpnn_loss_grad(mgm_ctx *c, const float *b_hat, const float *p_hat, const float *dp_hat, const float *target,
                       double *loss, float *grads, float *prediction)
{
    try {
        MpnnState &M = state(c);
        cudaStream_t s = c->s;
        Level &L = c->L[0];
        DBuf<float> bh, ph, dh, tt;
        bh.upload(b_hat, M.n, s);
        ph.upload(p_hat, M.n, s);
        dh.upload(dp_hat, M.n, s);
        tt.upload(target, M.n, s);
        k_features_ds<<<blocks_for(M.n, 256), 256, 0, s>>>(M.n, bh.p, ph.p, dh.p, L.x.p, L.y.p, L.btag.p, M.feat.p);
        MGM_LAUNCHED();
        loss_and_grad(M, tt.p, s);
        double ls = 0;
        M.scal.download(c->h_pinned, 3, s);
        MGM_CUDA(cudaStreamSynchronize(s));
        ls = c->h_pinned[2];
        if (loss) *loss = ls;
        if (grads) M.grads.download(grads, kNumParams, s);
        if (prediction) M.y.download(prediction, M.n, s);
        MGM_CUDA(cudaStreamSynchronize(s));
        return MGM_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    }
}

// the network's inference pass (the one a step runs) on normalised inputs
int mgm_mpnn_predict(mgm_ctx *c, const float *b_hat, const float *p_hat, const float *dp_hat, float *prediction)
{
    try {
        MpnnState &M = state(c);
        MGM_REQUIRE(b_hat && p_hat && dp_hat && prediction, "mgm_mpnn_predict: null argument");
        cudaStream_t s = c->s;
        Level &L = c->L[0];
        DBuf<float> bh, ph, dh;
        bh.upload(b_hat, M.n, s);
        ph.upload(p_hat, M.n, s);
        dh.upload(dp_hat, M.n, s);
        k_features_ds<<<blocks_for(M.n, 256), 256, 0, s>>>(M.n, bh.p, ph.p, dh.p, L.x.p, L.y.p, L.btag.p, M.feat.p);
        MGM_LAUNCHED();
        forward(M, false, s);
        M.y.download(prediction, M.n, s);
        MGM_CUDA(cudaStreamSynchronize(s));
        return MGM_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    }
}

// runs nsteps fractional steps with the given Poisson mode, recording (b, p_prev, p_new) samples
int mgm_mpnn_collect(mgm_ctx *c, int mode, int nsteps)
{
    try {
        MpnnState &M = state(c);
        MGM_REQUIRE(M.ds_cap > 0, "mgm_mpnn_collect: dataset capacity is zero");
        MGM_REQUIRE(mode == MGM_MODE_FP64 || mode == MGM_MODE_FP32_IR, "mgm_mpnn_collect: solver mode");
        DBuf<double> pprev(M.n), pprev2(M.n);
        for (int t = 0; t < nsteps; t++) {
            if (t > 0)
                MGM_CUDA(cudaMemcpyAsync(pprev2.p, pprev.p, sizeof(double) * M.n, cudaMemcpyDeviceToDevice, c->s));
            MGM_CUDA(cudaMemcpyAsync(pprev.p, c->L[0].p.p, sizeof(double) * M.n, cudaMemcpyDeviceToDevice, c->s));
            int st = mgm_step(c, mode, nullptr);
            if (st != MGM_OK) return st;
            record_sample(c, c->bvec.p, pprev.p, t > 0 ? pprev2.p : nullptr, c->L[0].p.p, c->s);
        }
        MGM_CUDA(cudaStreamSynchronize(c->s));
        return MGM_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    }
}

int mgm_mpnn_dataset_size(mgm_ctx *c, int *count)
{
    try {
        MpnnState &M = state(c);
        *count = std::min(M.ds_count, M.ds_cap);
        return MGM_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    }
}

// Adam on samples [first, first + count) of the dataset, `iters` iterations in a
// seeded shuffled order; losses[it] (host, may be NULL) receives each iteration's loss.
int mgm_mpnn_train(mgm_ctx *c, int first, int count, int iters, float lr, unsigned long long seed, double *losses)
{
    try {
        MpnnState &M = state(c);
        const int have = std::min(M.ds_count, M.ds_cap);
        MGM_REQUIRE(first >= 0 && count >= 1 && first + count <= have, "mgm_mpnn_train: sample range out of the dataset");
        cudaStream_t s = c->s;
        Level &L = c->L[0];
        DBuf<double> dl(std::max(iters, 1));
        dl.zero(s);
        unsigned long long x = seed * 0x9E3779B97F4A7C15ULL + 7;
        for (int it = 0; it < iters; it++) {
            x ^= x << 13; x ^= x >> 7; x ^= x << 17;
            const int smp = first + (int)(x % (unsigned long long)count);
            const float *slot = M.ds.p + (size_t)smp * kSlot * M.n;
            k_features_ds<<<blocks_for(M.n, 256), 256, 0, s>>>(M.n, slot, slot + M.n, slot + 2 * M.n, L.x.p, L.y.p,
                                                               L.btag.p, M.feat.p);
            MGM_LAUNCHED();
            loss_and_grad(M, slot + 3 * M.n, s);
            MGM_CUDA(cudaMemcpyAsync(dl.p + it, M.scal.p + 2, sizeof(double), cudaMemcpyDeviceToDevice, s));
            adam_step(M, lr, s);
        }
        if (losses && iters > 0) dl.download(losses, iters, s);
        MGM_CUDA(cudaStreamSynchronize(s));
        return MGM_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    }
}

// mean loss of the network on samples [first, first + count) (no update)
int mgm_mpnn_eval(mgm_ctx *c, int first, int count, double *mean_loss)
{
    try {
        MpnnState &M = state(c);
        const int have = std::min(M.ds_count, M.ds_cap);
        MGM_REQUIRE(first >= 0 && count >= 1 && first + count <= have, "mgm_mpnn_eval: sample range out of the dataset");
        cudaStream_t s = c->s;
        Level &L = c->L[0];
        DBuf<float> dyv(M.n);
        double tot = 0;
        for (int q = first; q < first + count; q++) {
            const float *slot = M.ds.p + (size_t)q * kSlot * M.n;
            k_features_ds<<<blocks_for(M.n, 256), 256, 0, s>>>(M.n, slot, slot + M.n, slot + 2 * M.n, L.x.p, L.y.p,
                                                               L.btag.p, M.feat.p);
            MGM_LAUNCHED();
            forward(M, false, s);
            loss_head(M, slot + 3 * M.n, s);
            M.scal.download(c->h_pinned, 3, s);
            MGM_CUDA(cudaStreamSynchronize(s));
            tot += c->h_pinned[2];
        }
        *mean_loss = tot / count;
        return MGM_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    }
}

int mgm_mpnn_set_loss(mgm_ctx *c, float w_mse, float w_res)
{
    try {
        MpnnState &M = state(c);
        MGM_REQUIRE(w_mse >= 0 && w_res >= 0 && w_mse + w_res > 0, "mgm_mpnn_set_loss: weights must be >= 0, not both 0");
        M.w_mse = w_mse;
        M.w_res = w_res;
        return MGM_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    }
}

int mgm_set_warm_start(mgm_ctx *c, int enable)
{
    try {
        MGM_REQUIRE(c, "null context");
        if (enable) {
            state(c);  // a network must exist
            c->guess_flags |= MGM_GUESS_LEARNED;
        } else {
            c->guess_flags &= ~MGM_GUESS_LEARNED;
        }
        return MGM_OK;
    } catch (const Error &e) {
        set_error(e.code, e.msg);
        return e.code;
    }
}

}  // extern "C"
