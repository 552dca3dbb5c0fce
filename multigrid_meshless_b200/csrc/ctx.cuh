// ctx.cuh -- the per-level device data and the solver context behind the C ABI.
#pragma once
#include "../../include/mgm.h"
#include "krylov.cuh"
#include "stencil.cuh"

namespace mgm {

struct MpnnState;  // learned warm start (mpnn.cu)

struct Level {
    int n = 0, nb = 0, k = 0, poly = 0, np = 0;
    double d_avg = 0;
    DBuf<double> x, y, z, nx, ny, nz;
    DBuf<uint8_t> btag;
    DBuf<int> cloud;  // row-major [n][k] after the reorder
    DBuf<int> idx;    // ELL [k][n]
    DBuf<double> Dx, Dy, Dz, lap, lapP;  // ELL
    DBuf<int> rpts, ppts;
    // reference-semantics transfer rows (rows >= nb), ELL
    DBuf<int> ref_r_idx, ref_p_idx;
    DBuf<double> ref_restr, ref_prol;
    // solver transfer: restriction into this level (interior rows), prolongation into this level (all rows)
    DBuf<int> s_r_idx, s_p_idx;
    DBuf<double> s_r_w64, s_p_w64;
    DBuf<float> s_r_w32, s_p_w32;
    // pinned operator: FP64 in the level's slot order [k][n]; FP32 with each
    // row's slots sorted by neighbour index, [k][ld4] (rows padded to a
    // multiple of 4 with zero weights), indices in sidx
    DBuf<double> A64, dinv64;
    DBuf<double> A64s;  // FP64 copy in the sorted slot order of A32, [k][ld4] (compact FP64 V-cycle)
    DBuf<float> A32, dinv32;
    DBuf<int> sidx;
    int ld4 = 0;
    DBuf<int> bnd_list;
    DBuf<int> bnd_idx;           // boundary rows' stencils, row-major [nbl][k]
    DBuf<double> bnd_A64;
    DBuf<float> bnd_A32;
    int nbl = 0;
    double lmax = 2.0;
    // compact FP32-path indices (int16 offsets): off16 [k][ld4] (sorted slots), r_off16/p_off16 [k][n]
    DBuf<short> off16, r_off16, p_off16;
    bool off_ok = false, r_off_ok = false, p_off_ok = false;
    // the compact operator again, tile-major ([ld / kTileRows][k][kTileRows],
    // rows padded to ld), streamed tile by tile into shared memory by bulk copies
    DBuf<float> A32t;
    DBuf<short> off16t;
    int ldt = 0;
    // FP16 operator of the half-operator V-cycle (levels of kVecMinRows rows
    // or more): D^-1 A (row sum in the diagonal slot) packed with the offsets,
    // four interleaved rows per uint4, [k][ldi / 4]
    int ldi = 0;
    DBuf<uint4> W16;
    bool h_ok = false;
    // reference-mode state
    DBuf<double> p, ptmp, src, res;
    // solver work vectors
    DBuf<double> r64, e64, e64b, d64, q64;
    DBuf<float> r32, e32, e32b, d32, q32;
};

}  // namespace mgm

using namespace mgm;

struct mgm_ctx {
    mgm::MpnnState *mpnn = nullptr;
    int dim = 2, phs = 3, nl = 0;
    int device = 0;
    cudaStream_t s = nullptr;
    std::vector<Level> L;
    bool setup_done = false;
    bool have_ref_transfer = false;
    // flow
    double Re = 100, courant = 0.5, dt = 0, nu = 0.01, rho = 1;
    float omega = 1.0f;
    int num_relax = 3, num_vcycles = 10;
    // level-0 fields
    DBuf<double> u, v, w, u_new, v_new, w_new, dpdn, partial, scal;
    // TIMPLE state (timple_solver.h): previous time level, pressure, gradients,
    // and the previous-sweep copies of the momentum iterations
    DBuf<double> u_old, v_old, w_old, p_old, dpdx, dpdy, dpdz, tu, tv, tw;
    int iter_timple = 1, iter_momentum = 1;
    // heat-conduction program (mgm_heat_init)
    int heat_wave = 0;
    bool heat_ready = false;
    double facRe = 1.0, facdt = 1.0;
    // solver controls and state
    double tol = 1e-8;
    int max_iters = 60, cheb_deg = 3;
    double cheb_ratio = 6.0;
    DBuf<double> cinv64;
    DBuf<float> cinv32;
    DBuf<double> V, Z64, wv, kpart, kscal, bvec, wdir;
    DBuf<float> Z32;
    int last_iters = 0;
    double last_relres = 0;
    long long vcycles_in_solve = 0;   // V-cycles of the last solve
    double last_learned_alpha = 0;    // step length the last solve took along the learned direction
    int warm_smooth_steps = 3;        // Chebyshev steps that clean the learned direction
    int guess_flags = 0;              // MGM_GUESS_* of the steps' solves
    // pressure history of the fractional steps: p at the start of the running
    // step's solve, the previous one (p_prev2 of the next step) and whether
    // that one exists (device flag, cleared by mgm_apply_bc)
    DBuf<double> p_start, p_hist;
    DBuf<int> hist_ok;
    bool use_tma = false;             // tile-streamed level kernels where a level has them (else 4 rows per thread)
    bool half_operator = false;       // FP32 V-cycle reads the FP16 operator where built
    bool chain_launches = true;       // V-cycle kernels after the first use programmatic dependent launch
    bool fused_coarse = false;        // levels below kVecMinRows rows in one cooperative V-cycle launch (opt-in: slower here)
    int fused_blocks = 0;             // its CTAs (one per SM)
    DBuf<unsigned> fused_bar;         // its grid barrier {arrivals, generation}
    // compatible right-hand sides (mgm_set_compatible_rhs): the pinned solution
    // for the interior indicator and {rho0(w), rho0(b)} on the device
    bool compat = false, compat_ready = false;
    DBuf<double> compat_pw, compat_s;
    bool warm_suspended = false;      // no learned warm start in the solve for p_w
    DBuf<int> tma_err;                // set by a tile-streamed kernel whose bounded wait ran out
    double *h_pinned = nullptr;
    SmootherProfile prof;
    // captured V-cycles, [0] FP64, [1] FP32 (re-captured when solver settings change)
    struct VGraph {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t x = nullptr;
        void *out = nullptr;        // level-0 correction buffer the graph writes
        bool prof = false;          // graph records smoother events
        size_t ev_first = 0, ev_pairs = 0;
        long long kernels = 0;      // kernel nodes in the graph
    } vg[2];
    bool use_graphs = true;
    // The device-resident state of the outer FGMRES (krylov.cuh), a pinned
    // host copy of its head, and the side streams that capture the bodies of
    // the solve's conditional WHILE nodes.
    DBuf<FgState> fg;
    FgState *h_fg = nullptr;
    cudaStream_t s_body[2] = {nullptr, nullptr};
    // A whole fractional step captured as one graph, [0] FP64, [1] FP32-IR:
    // momentum, divergence, the Poisson solve with its loops as conditional
    // nodes, the velocity correction and the steady-state error read-back.
    // Kernel nodes per replay = top + outer * restart cycles + inner * V-cycles.
    struct StepGraph {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t x = nullptr;
        int guess = 0;
        bool compat = false;
        double dt = 0;
        long long k_top = 0, k_outer = 0, k_inner = 0;
    } sg[2];
    bool step_graphs = true;  // mgm_step / mgm_run_steps replay the step graph (when not profiling)
    bool compact = true;    // FP32 V-cycle on compact storage
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    double poisson_ms_acc = 0;
    long long vcycles_acc = 0;
    long long ref_vcycles_acc = 0;    // reference-mode V-cycles of the running batch of steps
};

