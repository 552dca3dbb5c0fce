// batch.cuh -- hierarchies with per-node stencil sizes, their one-launch
// weight assembly, and the multi-right-hand-side V-cycle behind the
// mgm_batch_* entry points of include/mgm.h.
//
// The reference has one stencil size per level (structures.h:15-78); here a
// node's stencil size k_i may vary (with the level and the distance to the
// boundary), so the operators are stored as CSR: row i holds the first k_i
// entries of the node's k_max-nearest list (self first; boundary rows [i]
// followed by interior nodes, kdtree_functions.h:141-149).  Vectors of the
// multi-RHS solve are node-major [n][B] (B right-hand sides contiguous per
// node), so one gathered neighbour is one coalesced 32-lane access and each
// stencil weight is read once for all B right-hand sides.
#pragma once
#include <vector>

#include "../../include/mgm.h"
#include "krylov.cuh"
#include "weights.cuh"

namespace mgm {

constexpr int kBatchMaxLevels = 8;
constexpr int kBatchCta = 256;  // threads of the persistent weight-solve CTA

struct BLevel {
    int n = 0, nb = 0, poly = 0, np = 0, kmax = 0;
    DBuf<double> x, y, z, nx, ny, nz;
    DBuf<uint8_t> btag;
    DBuf<int> kk;      // stencil size per node
    DBuf<int> cloud;   // row-major [n][kmax] nearest list after the reorder
    DBuf<int> rp, col; // CSR structure of the level's operators
    long long nnz = 0;
    DBuf<double> Dx, Dy, Dz, lap, lapP;
    DBuf<int> rpts, ppts;
    // restriction into this level (rows of this level; boundary rows empty),
    // prolongation into this level (every row)
    DBuf<int> r_rp, r_col, p_rp, p_col;
    DBuf<double> r_w64, p_w64;
    DBuf<float> r_w32, p_w32;
    long long r_nnz = 0, p_nnz = 0;
    // pinned solve operator (row 0 -> p[0] = 0)
    DBuf<double> A64, dinv64;
    DBuf<float> A32, dinv32;
    DBuf<int> bnd_list;
    int nbl = 0;
    double lmax = 2.0;
    std::vector<int> h_kk;  // host copy of kk (task list)
};

// One autotuned size class of the weight batch.
struct BatchClass {
    int N = 0;             // system order k + np
    long long count = 0;   // systems of this order
    int team = 0;          // threads per system
    double us_per_system = 0;
};

// Multi-RHS work buffers of one level, precision T, [n][B].
template <class T>
struct BVecs {
    DBuf<T> r, e, e2, d, q;
};

}  // namespace mgm

struct mgm_batch {
    int dim = 2, phs = 3, nl = 0, device = 0;
    cudaStream_t s = nullptr;
    mgm::BLevel L[mgm::kBatchMaxLevels];
    bool setup_done = false;
    // weight batch record
    std::vector<mgm::BatchClass> classes;
    double weights_ms = 0, tuning_ms = 0;
    long long systems = 0;
    int tiles = 0, smem_bytes = 0, ctas_per_sm = 0;
    // solver settings
    double tol = 1e-8, cheb_ratio = 20.0;
    int restart = 24, max_restarts = 8, cheb_deg = 3;
    mgm::DBuf<double> cinv64;
    mgm::DBuf<float> cinv32;
    // multi-RHS buffers (sized for B right-hand sides)
    int B = 0;
    mgm::BVecs<double> v64[mgm::kBatchMaxLevels];
    mgm::BVecs<float> v32[mgm::kBatchMaxLevels];
    mgm::DBuf<double> X, Bv, V, part, hsc;
    mgm::DBuf<double> stage;  // right-hand sides / solutions in the caller's [nrhs][n] order, kept across solves
    mgm::DBuf<float> Z32;
    mgm::DBuf<double> Z64;
    int V_cols = 0, Z_cols32 = 0, Z_cols64 = 0;
    double *h_pinned = nullptr;
    size_t h_pinned_n = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
};

namespace mgm {
void batch_setup(mgm_batch *b, bool autotune);
void batch_prepare_solver(mgm_batch *b);
void batch_solve(mgm_batch *b, int mode, int nrhs, const double *rhs_host, double *sol_host, int *vcycles,
                 double *rel_res, double *solve_ms);
void batch_free_solver(mgm_batch *b);
}  // namespace mgm
