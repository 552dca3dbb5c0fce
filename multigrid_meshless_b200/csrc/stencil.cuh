// stencil.cuh -- argument blocks of the stencil and solver kernels.
#pragma once
#include <cuda_fp16.h>

#include "mgm_internal.cuh"

namespace mgm {

// level-0 state of one fractional step (device pointers; operators ELL [k][n])
struct StepArgs {
    int n, k;
    const int *idx;
    const double *Dx, *Dy, *Dz, *lap;
    const uint8_t *btag;
    const double *nx, *ny, *nz;
    double *u, *v, *w, *u_new, *v_new, *w_new;
    double *p, *source, *dpdn;
    double dt, nu, rho;
};

void launch_momentum(const StepArgs &a, int dim, cudaStream_t s);
void launch_divergence(const StepArgs &a, int dim, cudaStream_t s);
void launch_correct(const StepArgs &a, int dim, double *partial, double *d_err, cudaStream_t s);
void launch_mass_diag(const StepArgs &a, int dim, double *partial, double *d_out, cudaStream_t s);

// one level of the reference-semantics multigrid
struct RefLevel {
    int n, k;
    const int *idx;
    const double *lap, *lapP;
    const uint8_t *btag;
    double *p, *ptmp, *src, *res;
    // restriction into this level: gather index into the finer level's res (ELL [k_fine][n])
    const int *r_idx;
    const double *restr;
    // prolongation into this level from the coarser level (ELL [k_coarse][n])
    const int *p_idx;
    const double *prol;
};

// Which program's multigrid routines: the fractional step's
// (fractional_step_solver.h:150-246), the TIMPLE solver's
// (timple_solver.h:203-339) or the heat-conduction program's
// (heat_conduction.h:24-113).
enum RefVariant : int { REF_FS = 0, REF_TIMPLE = 1, REF_HEAT = 2 };
void ref_relaxation(const RefLevel &L, double w1, double w2, int num_relax, cudaStream_t s, RefVariant v = REF_FS);
void ref_residual_interior(const RefLevel &L, cudaStream_t s, RefVariant v = REF_FS);
void ref_restrict(const RefLevel &F, const RefLevel &C, cudaStream_t s, RefVariant v = REF_FS);
void ref_prolongate(const RefLevel &F, const RefLevel &C, cudaStream_t s, RefVariant v = REF_FS);
void ref_multigrid(std::vector<RefLevel> &Ls, double w1, double w2, int num_relax, int num_vcycles, cudaStream_t s,
                   RefVariant v = REF_FS);

// ---------------------------------------------------------------------------
// convergent solver (solver.cu)
// ---------------------------------------------------------------------------
// One level of the preconditioning V-cycle in precision T.
template <class T>
struct SolveLevel {
    int n, k, nb_list;            // rows, stencil width, number of boundary rows
    int ld;                       // leading dimension of idx, A and off (>= n; a multiple of 4 on FP32 levels)
    const int *idx;               // ELL [k][ld]
    const T *A;                   // lap_Poison, row 0 replaced by the pin (A[0][0] = 1, rest 0)
    const T *dinv;                // 1 / diagonal
    const uint8_t *btag;
    const int *bnd_list;          // boundary rows (incl. the pinned row 0)
    const int *bnd_idx;           // their stencils, row-major [nb_list][k]
    const T *bnd_A;
    T *r, *e, *e2, *d, *q;        // rhs, correction (double-buffered), Chebyshev direction, residual
    // restriction into this level (coarse row i <- fine interior residual), ELL [kf][n]
    int kr;
    const int *r_idx;
    const T *r_w;
    // prolongation from the coarser level into this level (all rows), ELL [kc][n]
    int kp;
    const int *p_idx;
    const T *p_w;
    double lmax;                  // spectral radius estimate of D^-1 A on interior rows
    // compact indices (each used when non-null; A then holds each row's slots
    // sorted by neighbour index, [k][ld], ld a multiple of 4): neighbours as
    // int16 offsets c - i [k][ld]; transfer gathers as int16 offsets from a
    // per-row base node (restriction: rpts, prolongation: ppts)
    const short *off = nullptr;
    const short *r_off = nullptr;
    const int *r_base = nullptr;
    const short *p_off = nullptr;
    const int *p_base = nullptr;
    // tile-streamed copy of (A, off), tile-major over ldt padded rows (FP32 path; used when non-null)
    const float *At = nullptr;
    const short *offt = nullptr;
    int ldt = 0;
    int *tma_err = nullptr;
    // FP16 copy of the compact operator (levels of at least kVecMinRows rows;
    // used when non-null): D^-1 A with the row sum in the diagonal slot, one
    // uint4 {4 FP16 weights, 4 int16 offsets} per slot and thread, the
    // thread's rows interleaved (128 g + 32 v + lane), [k][ldi / 4] with ldi
    // the rows rounded up to a multiple of 128
    const uint4 *W16 = nullptr;
    int ldi = 0;
};

// rows from which a compact level runs the four-rows-per-thread kernels
// (below: one row per thread); the FP16 operator is built from here too
constexpr int kVecMinRows = 65536;

// rows per tile of the tile-streamed level kernels
constexpr int kTileRows = 256;
// smallest level the tile-streamed kernels are used on (smaller levels fit in L2)
constexpr int kTileMinRows = 65536;
// largest stencil width the tile-streamed kernels take (two stages of k x 1.5 KB in shared memory)
constexpr int kTileMaxK = 64;

template <class T>
struct CoarseSolve {
    int n;
    const T *inv;  // dense inverse of the pinned coarsest operator, row-major [n][n]
};

// Records CUDA events around the level-0 Chebyshev kernels (the dominant
// kernel of a solve) so that their device time can be read back.
// In a captured CUDA graph the same event pairs are re-recorded on every
// replay: harvest_graph() reads them without releasing them.
struct SmootherProfile {
    bool on = false;
    std::vector<cudaEvent_t> ev;  // pairs
    size_t used = 0;
    double ms = 0;
    long long launches = 0;
    void mark(cudaStream_t s);    // records the next event of a pair
    void harvest();               // accumulates finished pairs (stream must be idle)
    void harvest_graph(size_t first, size_t pairs);  // accumulates pairs recorded by a graph replay
    ~SmootherProfile();
};

// the fused coarse-level V-cycle's launch: CTAs (one per SM), its grid
// barrier {arrivals, generation} and the flag a timed-out barrier sets
struct FusedCtl {
    bool on = false;
    int blocks = 0;
    unsigned *bar = nullptr;
    int *err = nullptr;
};
int fused_vcycle_blocks();
cudaError_t launch_coop_probe(cudaStream_t s);
cudaError_t launch_barrier_selftest(cudaStream_t s, unsigned *bar, int *err);

// chain: launch the kernels after the first with programmatic stream
// serialisation (Chain in mgm_internal.cuh); fused (when on): the levels
// below kVecMinRows rows run as one cooperative launch (k_coarse_vcycle)
template <class T>
void vcycle(std::vector<SolveLevel<T>> &Ls, const CoarseSolve<T> &cs, int cheb_degree, double cheb_ratio,
            cudaStream_t s, SmootherProfile *prof = nullptr, bool chain = false, const FusedCtl *fused = nullptr);
template <class T>
void estimate_lmax(SolveLevel<T> &L, cudaStream_t s);
template <class T>
const T *smooth_from_zero(SolveLevel<T> &L, int degree, double ratio, cudaStream_t s, bool chain = false);

}  // namespace mgm
