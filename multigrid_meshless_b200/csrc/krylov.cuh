// krylov.cuh -- FP64 vector kernels of the outer flexible GMRES and the set-up dense inverse.
#pragma once
#include <algorithm>
#include <cstddef>

#include "mgm_internal.cuh"

namespace mgm {

constexpr int kMaxKrylov = 128;

void resid64(int n, int k, const int *idx, const double *A, const double *b, const double *x, double *r, double *part,
             cudaStream_t s);
template <class T>
void apply64(int n, int k, const int *idx, const double *A, const T *z, double *w, cudaStream_t s);
int dot_blocks(int n);
void multidot(int n, int cnt, const double *V, long ldv, const double *w, double *part, double *out, cudaStream_t s);
void reduce_parts(const double *part, int nblk, int cnt, double *out, cudaStream_t s);
void orth_update(int n, int cnt, const double *V, long ldv, const double *h, double *w, cudaStream_t s);
// w -= sum_c h[c] V_c and *norm2 = |w|^2 of the result (device scalar)
void orth_norm(int n, int cnt, const double *V, long ldv, const double *h, double *w, double *part, double *norm2,
               cudaStream_t s);
void scale_by(int n, const double *in, double *out, const double *nrm, int is_sq, cudaStream_t s);
template <class T>
void combine(int n, int cnt, const T *Z, long ldz, const double *y, double *x, cudaStream_t s);
template <class T>
void copy_convert(long n, const double *in, T *out, cudaStream_t s);
template <class T>
void copy_out(long n, const T *in, T *out, cudaStream_t s);
void dense_inverse(int n, int k, const int *idx, const double *A, double *inv64, float *inv32, cudaStream_t s);

// ---------------------------------------------------------------------------
// Device-resident control of the outer flexible GMRES.  Every scalar of the
// iteration (norms, Gram-Schmidt projections, the Hessenberg matrix, Givens
// rotations, the convergence tests) lives here and is updated by small
// kernels, so that the whole solve can run inside one CUDA graph: the two
// loops (restart cycles, Arnoldi steps) are either WHILE conditional nodes
// whose conditions these kernels set, or host loops that read go_outer /
// go_inner after each pass (the same kernels in the same order, so the two
// forms give the same bits).
// ---------------------------------------------------------------------------
enum FgStatus { FG_OK = 0, FG_NONFINITE = 1, FG_NOT_CONVERGED = 2 };

struct FgState {
    // scalars first: the host loops read only this head (kFgHead bytes)
    double nrm;                 // |w|^2 after the last Gram-Schmidt pass
    double beta, bnorm, relres, alpha;
    double tol;
    int m, max_total, max_restarts;
    int j, j_done, total_it, restarts, vcycles;
    int reorth;
    int go_outer, go_inner;
    int status;
    // accumulated over solves until fg_clear_totals
    int err_any;                // bit 0: non-finite residual, bit 1: tolerance not reached
    int pad_;
    long long vcycles_total;    // Arnoldi steps (V-cycles)
    long long cycles_total;     // restart cycles begun
    long long solves_total;
    unsigned long long t_mark;  // %globaltimer at the last start mark
    unsigned long long t_ns;    // summed ns between start and end marks
    double start_log_relres;    // summed log10 of each solve's starting relative residual (after its guess)
    double head_end_;
    // arrays
    double H[(kMaxKrylov + 1) * kMaxKrylov];  // column j at H[j * (m + 1)]
    double cs[kMaxKrylov], sn[kMaxKrylov], g[kMaxKrylov + 1], y[kMaxKrylov];
    double h[kMaxKrylov + 2];   // projections of the first Gram-Schmidt pass (h[j+1] = |w|^2)
    double h2[kMaxKrylov + 2];  // projections of the re-orthogonalisation (0 when skipped)
};
constexpr size_t kFgHead = offsetof(FgState, H);

// handles of the two WHILE nodes when the solve is captured (0: host loops)
struct FgHandles {
    cudaGraphConditionalHandle outer = 0, inner = 0;
    int use = 0;
};

void fg_init(FgState *st, int m, int max_total, int max_restarts, double tol, cudaStream_t s);
void fg_clear_totals(FgState *st, cudaStream_t s);
void fg_time_mark(FgState *st, int end, cudaStream_t s);
void fg_begin(FgState *st, const double *part, int nbres, FgHandles hd, cudaStream_t s);
void fg_scale0(int n, double *V, const FgState *st, cudaStream_t s);
template <class T>
void fg_load(int n, const double *V, long ld, const FgState *st, T *out, cudaStream_t s);
template <class T>
void fg_store(int n, const T *z, T *Z, long ld, const FgState *st, cudaStream_t s);
template <class T>
void fg_apply(int n, int k, const int *idx, const double *A, const T *Z, long ld, const FgState *st, double *V,
              cudaStream_t s);
// one Gram-Schmidt pass against V_0..V_j (pass 0: projections and |w|^2 of
// V_0..V_{j+1}; pass 1, run only when the first asked for it: V_0..V_j) and
// the update w -= sum h V with the new |w|^2
void fg_gram_schmidt(int n, double *V, long ld, FgState *st, int pass, double *part, cudaStream_t s);
void fg_dgks(FgState *st, cudaStream_t s);
void fg_scale_w(int n, double *V, long ld, const FgState *st, cudaStream_t s);
void fg_arnoldi_end(FgState *st, FgHandles hd, cudaStream_t s);
void fg_solve_y(FgState *st, FgHandles hd, cudaStream_t s);
template <class T>
void fg_combine(int n, const T *Z, long ld, const FgState *st, double *x, cudaStream_t s);
void fg_final(FgState *st, cudaStream_t s);
// initial guess: coefficients c minimising |r0 - sum_i c_i AD_i|_2 over nd (1 or
// 2) directions from ks[i] = AD_i . r0, ks[2 + i] = AD_i . AD_0, ks[4 + i] =
// AD_i . AD_1, into ks[6 + i]; a zero or collinear direction is dropped; the
// coefficient of the last direction into st->alpha
void fg_guess_coefficients(FgState *st, double *ks, int nd, cudaStream_t s);
void set_scalar(double *dst, double v, cudaStream_t s);

}  // namespace mgm
