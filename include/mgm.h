/*
 * mgm.h -- C ABI of the B200 (sm_100a) meshless RBF-FD multigrid hot path.
 *
 * Plain C types only (no torch, no C++), so any host language that can call C
 * can bind it (ctypes, cgo, JNI, N-API).  Every entry point returns an int
 * status (MGM_OK or an MGM_ERR_* code) unless it returns a handle; the text of
 * the last failure in the calling thread is available from mgm_last_error().
 *
 * Layout conventions at the boundary (host memory):
 *   - node arrays: length n, in the level's node order;
 *   - stencil arrays (cloud indices and operator weights): row-major [n][k],
 *     i.e. the reference's jagged `int**` / `double**` rows laid end to end;
 *   - boundary tags: one byte per node, non-zero = boundary.
 *
 * Each declaration cites the reference function it replaces
 * (Multigrid_meshless, path within that project : line).
 */
#ifndef MGM_H
#define MGM_H

#include <stddef.h>

#if defined(__GNUC__)
#define MGM_API __attribute__((visibility("default")))
#else
#define MGM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define MGM_OK 0
#define MGM_ERR_CUDA 1      /* a CUDA call failed (message holds the CUDA error) */
#define MGM_ERR_ARG 2       /* invalid argument or input (e.g. disconnected stencil graph) */
#define MGM_ERR_DIVERGED 3  /* NaN/Inf or growth in a residual */
#define MGM_ERR_TIMEOUT 4   /* a bounded device-side wait ran out */
#define MGM_ERR_NOMEM 5     /* device allocation failed */
#define MGM_ERR_STATE 6     /* call made in the wrong state (e.g. before set-up) */

/* ------------------------------------------------------------------ */
/* Diagnostics                                                         */
/* ------------------------------------------------------------------ */
MGM_API const char *mgm_last_error(void);
/* Makes `device` the current CUDA device of the calling thread for this
 * library (contexts are created on the current device). */
MGM_API int mgm_set_device(int device);
/* Number of kernels this library has launched in the calling process. */
MGM_API long long mgm_kernel_launches(void);
MGM_API int mgm_version(void);

/* ------------------------------------------------------------------ */
/* Mesh files                                                          */
/* ------------------------------------------------------------------ */
typedef struct mgm_mesh mgm_mesh;
/* read_PointStructure (header_files/mesh_functions.h:172-476): reads a Gmsh
 * 2.2 ASCII mesh as one level's nodes in the state the reference's reader
 * leaves them -- boundary tags and unnormalised normals accumulated from the
 * boundary elements (2D: 2-node lines; 3D: 3-node triangles and 4-node
 * quads), corner nodes (1-node points; in 3D also both ends of 2-node lines)
 * counted and the first that many nodes dropped, d_avg from the bounding box
 * and the element count.  The normals are summed on the calling thread's
 * current device.  Unreadable or malformed files give MGM_ERR_ARG (the
 * reference prints and exits). */
MGM_API int mgm_mesh_read(const char *path, int dim, mgm_mesh **mesh);
/* num_nodes (after the corner removal), num_boundary_nodes (corners
 * subtracted, as the reference does), num_elem, d_avg; any may be NULL. */
MGM_API int mgm_mesh_info(const mgm_mesh *mesh, int *num_nodes, int *num_boundary_nodes, int *num_elem,
                          double *d_avg);
/* Copies num_nodes entries into each non-NULL array. */
MGM_API int mgm_mesh_get(const mgm_mesh *mesh, double *x, double *y, double *z, double *nx, double *ny, double *nz,
                         unsigned char *boundary_tag, unsigned char *corner_tag);
MGM_API void mgm_mesh_free(mgm_mesh *mesh);

/* ------------------------------------------------------------------ */
/* Stateless set-up operations: host arrays in, host arrays out.       */
/* Each call uploads its inputs, runs its kernels and downloads the    */
/* result (the reference's own call shape).                            */
/* ------------------------------------------------------------------ */

/* find_cloud_index (header_files/kdtree_functions.h:113-151).
 * Nodes i >= nb: the k nearest nodes (self first).  Nodes i < nb: cloud[i][0]
 * = i followed by the k-1 nearest nodes whose btag is 0.  Distances are the
 * reference's sqrt(((dx*dx)+dy*dy)+dz*dz) (kdtree_functions.h:28-35, 84);
 * exactly equal distances are ordered by lower node index. */
MGM_API int mgm_knn_cloud(int n, int nb, int dim, const double *x, const double *y, const double *z,
                  const unsigned char *btag, int k, int *cloud);

/* find_nearest_point (header_files/kdtree_functions.h:153-175) with
 * num_cloud_points = 1: for each node of set 1, the nearest node of set 2. */
MGM_API int mgm_nearest_points(int n1, const double *x1, const double *y1, const double *z1,
                       int n2, const double *x2, const double *y2, const double *z2, int dim, int *nearest);

/* rcm_reordering_with_boundarynodes (header_files/mesh_functions.h:774-872):
 * FIFO breadth-first order from node 0 over cloud slots 1..k-1.  queue1[i] =
 * old index of new node i.  Returns MGM_ERR_ARG if the stencil graph is
 * disconnected (the reference leaves the tail of its queue uninitialised). */
MGM_API int mgm_bfs_order(int n, int k, const int *cloud, int *queue1);

/* The permutation step of rcm_reordering_with_boundarynodes
 * (mesh_functions.h:821-855), in place: coordinates, normals, boundary tags
 * and cloud rows gathered through queue1, cloud entries renumbered. */
MGM_API int mgm_apply_order(int n, int k, const int *queue1, double *x, double *y, double *z,
                    double *nx, double *ny, double *nz, unsigned char *btag, int *cloud);

/* correct_normal_directions (header_files/mesh_functions.h:478-527), in place. */
MGM_API int mgm_correct_normals(int n, int k, const double *x, const double *y, const double *z,
                        const unsigned char *btag, const int *cloud, double *nx, double *ny, double *nz);

/* calculate_avg_dx (header_files/mesh_functions.h:895-910). */
MGM_API int mgm_avg_dx(int n, int k, int dim, const double *x, const double *y, const double *z,
               const unsigned char *btag, const int *cloud, double *d_avg);

/* No counterpart in the reference.  mgm_avg_dx for callers that cannot let a
 * library allocate device memory (their device memory is owned by another
 * allocator or a fixed arena, or they cannot afford cudaMalloc's device-wide
 * synchronisation).  All pointers are DEVICE pointers owned by the caller:
 * coordinates and tags [n], cloud row-major [n][k], d_avg one double.  Runs
 * asynchronously on `stream` (a cudaStream_t; NULL = the legacy default
 * stream) and calls no cudaMalloc/cudaFree: its scratch is a fixed device
 * array of MGM_NOALLOC_MAX_NODES doubles (16 MiB) that every GPU loading this
 * library keeps until exit.  n above that limit is rejected with MGM_ERR_ARG.
 * The first call on a device looks up the array's device address; make that
 * first call before any stream capture.  `stream` must belong to the device
 * that is current at the call (the address looked up is that device's).  The
 * address is kept for the life of the process, so cudaDeviceReset after the
 * first call is not supported.  Calls share the array: calls that overlap on
 * the GPU race. */
#define MGM_NOALLOC_MAX_NODES 2097152
MGM_API int mgm_avg_dx_noalloc(int n, int k, int dim, const double *d_x, const double *d_y, const double *d_z,
                               const unsigned char *d_btag, const int *d_cloud, double *d_avg, void *stream);

/* create_derivative_matrices (header_files/rbf.h:401-421) including
 * create_laplacian_for_Poisson (rbf.h:382-399).  Outputs [n][k]; Dz is only
 * written when dim == 3 (may be NULL otherwise). */
MGM_API int mgm_derivative_weights(int n, int k, int dim, int phs, int poly_degree,
                           const double *x, const double *y, const double *z,
                           const double *nx, const double *ny, const double *nz,
                           const unsigned char *btag, const int *cloud,
                           double *Dx, double *Dy, double *Dz, double *lap, double *lapP);

/* create_restriction_matrix / create_prolongation_matrix
 * (header_files/mesh_functions.h:533-600, 602-670): RBF interpolation weights
 * [nt][ks] from the source level's cloud around src_pt[i] to target node i.
 * Rows i < rows_from stay zero (the reference starts at num_boundary_nodes,
 * :563, :633); with only_interior != 0, rows with a boundary tag stay zero
 * instead and every other row is filled. */
MGM_API int mgm_transfer_weights(int nt, const double *tx, const double *ty, const double *tz,
                         const unsigned char *tbtag, const int *src_pt, int rows_from, int only_interior,
                         int ns, int ks, int dim, int phs, int poly_degree_src,
                         const double *sx, const double *sy, const double *sz, const int *scloud, double *W);

/* multiply_sparse_matrix_vector_gpu (header_files/mat_lib.h:80-89):
 * out[i] = sum_j D[i][j] * f[cloud[i][j]], j ascending, no fused multiply-add
 * (bit-identical to the reference's C build). */
MGM_API int mgm_spmv(int n, int k, const double *D, const int *cloud, const double *f, double *out);

/* matrixInverse_Gauss_Jordan (header_files/mat_lib.h:423-491) of one dense
 * row-major order x order matrix on the GPU: one bubble pass on column 0,
 * elimination without pivoting, rows scaled last, every operation rounded
 * separately (the same bits as the reference's C build).  order <= 1024. */
MGM_API int mgm_gauss_jordan(int order, const double *A, double *inverse);

/* create_laplacian_for_Poisson (header_files/rbf.h:382-399): lapP = lap on
 * interior rows, Dx nx + Dy ny (+ Dz nz in 3D) on boundary rows; [n][k]. */
MGM_API int mgm_laplacian_for_poisson(int n, int k, int dim, const double *Dx, const double *Dy, const double *Dz,
                                      const double *lap, const double *nx, const double *ny, const double *nz,
                                      const unsigned char *btag, double *lapP);

/* ------------------------------------------------------------------ */
/* Device-resident solver context (copyin_*_to_gpu + the time loop)    */
/* ------------------------------------------------------------------ */
typedef struct mgm_ctx mgm_ctx;

/* Creates a context on the current CUDA device.  dim 2 or 3, phs the
 * polyharmonic exponent (parameters.phs_degree, structures.h:19). */
MGM_API mgm_ctx *mgm_create(int dim, int phs_degree, int num_levels);
MGM_API void mgm_destroy(mgm_ctx *ctx);

/* Raw level input (the state read_PointStructure leaves, mesh_functions.h:172-476):
 * boundary nodes first (indices < nb), no corner nodes. */
MGM_API int mgm_set_level(mgm_ctx *ctx, int lev, int n, int nb, const double *x, const double *y, const double *z,
                  const double *nx, const double *ny, const double *nz, const unsigned char *btag,
                  int poly_degree, int k);

#define MGM_SETUP_REFERENCE_TRANSFER 1 /* also build the reference's transfer rows (rows >= nb only) */
/* Runs, on the GPU, read_complete_mesh_data's pipeline after the reader
 * (mesh_functions.h:914-928: kNN clouds, breadth-first reorder, normals,
 * average spacing, nearest points, restriction/prolongation weights) and
 * create_derivative_matrices on every level (rbf.h:401-421), then packs the
 * ELL operators and prepares the Poisson solver (coarsest-level inverse,
 * smoother bounds).  flags: MGM_SETUP_*. */
MGM_API int mgm_setup(mgm_ctx *ctx, int flags);

/* Loads a level whose set-up was done elsewhere (e.g. by the stateless calls
 * above into the reference's host structures): geometry after the reorder,
 * cloud [n][k], operators [n][k] (Dz only in 3D), restriction/prolongation
 * points and d_avg.  Then optionally the reference's transfer matrices
 * (restr [n][k of lev-1], prol [n][k of lev+1]; NULL to skip), and
 * mgm_prepare() builds the solver's data (the copyin_*_to_gpu step,
 * openACC_functions.h:96-120). */
MGM_API int mgm_load_level(mgm_ctx *ctx, int lev, int n, int nb, const double *x, const double *y, const double *z,
                           const double *nx, const double *ny, const double *nz, const unsigned char *btag,
                           int poly_degree, int k, const int *cloud, const double *Dx, const double *Dy,
                           const double *Dz, const double *lap, const double *lapP, const int *rpts, const int *ppts,
                           double d_avg);
MGM_API int mgm_load_transfer(mgm_ctx *ctx, int lev, const double *restr, const double *prol);
MGM_API int mgm_prepare(mgm_ctx *ctx);

MGM_API int mgm_level_size(mgm_ctx *ctx, int lev, int *n, int *nb, int *k, int *num_poly_terms);
MGM_API int mgm_level_d_avg(mgm_ctx *ctx, int lev, double *d_avg);

/* Downloads a level after set-up (arrays sized by mgm_level_size; [n][k] row-major).
 * Any pointer may be NULL to skip it.  Dz only in 3D. */
MGM_API int mgm_get_geometry(mgm_ctx *ctx, int lev, double *x, double *y, double *z, double *nx, double *ny, double *nz,
                     unsigned char *btag, int *cloud);
MGM_API int mgm_get_operators(mgm_ctx *ctx, int lev, double *Dx, double *Dy, double *Dz, double *lap, double *lapP);
/* restriction_points / prolongation_points and the reference-semantics
 * restr_mat ([n][k of level lev-1]) / prol_mat ([n][k of level lev+1]). */
MGM_API int mgm_get_transfer(mgm_ctx *ctx, int lev, int *rpts, int *ppts, double *restr, double *prol);
/* The convergent solver's transfer weights of a level (no counterpart in the
 * reference): restriction into the level from level lev-1, built with
 * create_restriction_matrix's interpolation (mesh_functions.h:533-600) for
 * every non-boundary row ([n][k of level lev-1], boundary rows 0), and
 * prolongation into the level from level lev+1, built with
 * create_prolongation_matrix's interpolation (:602-670) for every row
 * ([n][k of level lev+1]).  Either pointer may be NULL. */
MGM_API int mgm_get_solver_transfer(mgm_ctx *ctx, int lev, double *restr, double *prol);
/* The FP32 V-cycle's compact copies of a level as the level kernels read
 * them, decoded (no counterpart in the reference).  which = 0: the pinned
 * operator with each row's slots sorted by neighbour index, [n][k]; 1: the
 * restriction into the level, [n][k of level lev-1]; 2: the prolongation
 * into the level, [n][k of level lev+1].  idx[i][j] is the gathered node:
 * rebuilt from the int16 offset (row i, restriction / prolongation point of
 * row i) where the level holds the offsets (*compact = 1), else the stored
 * 32-bit index (*compact = 0); w[i][j] the FP32 weight. */
MGM_API int mgm_get_compact(mgm_ctx *ctx, int lev, int which, int *idx, float *w, int *compact);

/* Flow parameters (read_flow_parameters, mesh_functions.h:37-100: rho = 1,
 * mu = rho/Re, nu = mu/rho).  dt <= 0 computes calculate_dt
 * (general_functions.h:34-41) from level 0's average spacing. */
MGM_API int mgm_set_flow(mgm_ctx *ctx, double Re, double courant, float omega, int num_relax, int num_vcycles, double dt);
MGM_API int mgm_get_dt(mgm_ctx *ctx, double *dt);

/* Level-0 fields.  which: MGM_FIELD_*.  Host arrays of length n(level). */
#define MGM_FIELD_U 0
#define MGM_FIELD_V 1
#define MGM_FIELD_W 2
#define MGM_FIELD_P 3
#define MGM_FIELD_U_NEW 4
#define MGM_FIELD_V_NEW 5
#define MGM_FIELD_W_NEW 6
#define MGM_FIELD_U_OLD 7
#define MGM_FIELD_V_OLD 8
#define MGM_FIELD_W_OLD 9
#define MGM_FIELD_RES 10
#define MGM_FIELD_SOURCE 11
#define MGM_FIELD_DPDN 12
#define MGM_FIELD_DPDX 13
#define MGM_FIELD_DPDY 14
#define MGM_FIELD_DPDZ 15
#define MGM_FIELD_P_OLD 16  /* TIMPLE pressure (the fractional step's pressure is MGM_FIELD_P) */
#define MGM_FIELD_PPRIME MGM_FIELD_P  /* TIMPLE: the level's pressure correction lives in the P buffer */
MGM_API int mgm_set_field(mgm_ctx *ctx, int lev, int which, const double *values);
MGM_API int mgm_get_field(mgm_ctx *ctx, int lev, int which, double *values);

/* Boundary/initial conditions on level 0: MGM_BC_LID (init/init_LDC.c:16-44)
 * or MGM_BC_TAYLOR_COUETTE (init/init_TC.c:17-54).  Every field of every
 * level (velocities and their copies, pressures, p', sources, residuals,
 * gradients) is zeroed first, as the reference's fields start. */
#define MGM_BC_LID 0
#define MGM_BC_TAYLOR_COUETTE 1
MGM_API int mgm_apply_bc(mgm_ctx *ctx, int kind);

/* time_implicit_solver (header_files/timple_solver.h:40-70), the default solver
 * of mg_NS_solver.c: iter_timple outer iterations of iter_momentum implicit
 * momentum sweeps (calculate_intermediate_velocity_implicit, :72-175), the mass
 * residual (:177-201), the pressure-correction solve, the velocity and pressure
 * update (:341-369) and the boundary pressure (:371-410).  Velocities live in
 * MGM_FIELD_U_NEW/V_NEW/W_NEW (the boundary conditions too), the pressure in
 * MGM_FIELD_P_OLD.  Momentum sweeps run in data-parallel order (every node from
 * the previous sweep's values; the reference's C build updates in place).  mode:
 * MGM_MODE_REFERENCE = the reference's fixed V-cycles on p' (timple variant,
 * :203-339); MGM_MODE_FP64 / MGM_MODE_FP32_IR = the convergent pinned solve. */
MGM_API int mgm_set_timple(mgm_ctx *ctx, int iter_timple, int iter_momentum, double facRe, double facdt);
MGM_API int mgm_timple_step(mgm_ctx *ctx, int mode, double *steady_err);
/* nsteps TIMPLE steps timed with CUDA events on the context's stream:
 * step_ms (all steps), vcycles (p' V-cycles over all steps), the last
 * steady-state error; any output may be NULL. */
MGM_API int mgm_timple_run(mgm_ctx *ctx, int mode, int nsteps, double *step_ms, long long *vcycles,
                           double *steady_err);
/* One part of a TIMPLE iteration, for callers that drive the loop themselves
 * (the reference's callees): */
#define MGM_TIMPLE_MOMENTUM 0           /* calculate_intermediate_velocity_implicit (:72-175) */
#define MGM_TIMPLE_MASS 1               /* calculate_mass_residual_implicit (:177-201) */
#define MGM_TIMPLE_PRESSURE 2           /* the p' solve (multigrid_Poisson_solver, :203-220, in `mode`) */
#define MGM_TIMPLE_UPDATE 3             /* update_velocity_implicit (:341-369) */
#define MGM_TIMPLE_BOUNDARY_PRESSURE 4  /* update_boundary_pressure (:371-410) */
MGM_API int mgm_timple_part(mgm_ctx *ctx, int part, int mode);

/* The heat-conduction program (mg_heat_conduction.c:43-83 with
 * header_files/heat_conduction.h:24-113 and init/init_heat_conduction.c:
 * 14-67), 2D, on a context set up with MGM_SETUP_REFERENCE_TRANSFER.
 * mgm_heat_init: initial_conditions, boundary_conditions and
 * set_boundary_rhs for wave number k: level-0 source
 * -8 pi^2 k^2 sin(2 pi k x) sin(2 pi k y) (pi written 3.14), every p and
 * residual 0, coarse sources 0; the boundary nodes with x == 0 become
 * Dirichlet rows (level 0's lap_Poison row = e_i, right-hand side 1 -- this
 * changes level 0's lap_Poison, as the reference does), the other boundary
 * nodes get the manufactured solution's normal derivative as right-hand side.
 * mgm_heat_step: one pass of the program's time loop -- num_vcycles of its own
 * V-cycles (omega, num_relax and num_vcycles of mgm_set_flow; sweeps in
 * data-parallel order) -- and *steady_err = sum over level 0 of the squared
 * change of p (the value the program compares with its steady-state
 * tolerance; it prints sqrt(sum / n)).  p is MGM_FIELD_P of each level. */
MGM_API int mgm_heat_init(mgm_ctx *ctx, int wave_number);
MGM_API int mgm_heat_step(mgm_ctx *ctx, double *steady_err);

/* Output and restart.
 * mgm_write_solution: Solution.csv as mg_NS_solver.c:83-88 writes it --
 * "%lf, %lf, %lf, %lf, %lf, %lf, %lf\n" of x, y, z, u, v, w and the pressure
 * field (MGM_FIELD_P_OLD, the TIMPLE pressure the reference main writes, or
 * MGM_FIELD_P), one line per level-0 node in the set-up's node order.
 * mgm_checkpoint_save / _load: every field one time step hands to the next
 * (each level's p, source and residual; level 0's velocities, their
 * intermediate and old copies, dp/dn, grad p, the TIMPLE pressure) in one
 * binary file, with the levels' sizes and a fingerprint of their coordinates
 * and a checksum; a context loads only a checkpoint of matching levels
 * (MGM_ERR_ARG otherwise), after mgm_setup (and after mgm_heat_init for the
 * heat-conduction program).  A run continued from a checkpoint repeats the
 * uninterrupted run bit for bit (with the default initial guess: the
 * pressure history of mgm_set_initial_guess is not saved, so the first step
 * after a load starts from the previous pressure alone).  No counterpart in
 * the reference. */
MGM_API int mgm_write_solution(mgm_ctx *ctx, const char *path, int pressure_field);
MGM_API int mgm_checkpoint_save(mgm_ctx *ctx, const char *path);
MGM_API int mgm_checkpoint_load(mgm_ctx *ctx, const char *path);

/* Poisson solve modes */
#define MGM_MODE_REFERENCE 0   /* multigrid_Poisson_solver semantics, fixed num_vcycles (Jacobi-order sweeps) */
#define MGM_MODE_FP64 1        /* convergent V-cycle preconditioned FGMRES, all FP64 */
#define MGM_MODE_FP32_IR 2     /* same, V-cycle in FP32 inside the FP64 FGMRES refinement */

/* fractional_step_explicit (header_files/fractional_step_solver.h:47-71):
 * momentum, divergence, boundary dp/dn, Poisson solve (mode), velocity
 * correction; *steady_err receives sqrt(sum |du|^2 / n).  For the solve modes
 * other than MGM_MODE_REFERENCE the Poisson solve runs to the relative
 * residual set by mgm_set_solver. */
MGM_API int mgm_step(mgm_ctx *ctx, int mode, double *steady_err);

/* Solver controls for MGM_MODE_FP64 / MGM_MODE_FP32_IR. */
MGM_API int mgm_set_solver(mgm_ctx *ctx, double rel_tol, int max_iters, int cheb_degree, double cheb_ratio);
/* MGM_MODE_FP32_IR preconditioner indices: compact (default; neighbour
 * indices as 16-bit offsets from the row, transfer gathers as 16-bit offsets
 * from the row's nearest node, wherever the reordered bandwidth allows) or
 * 32-bit (enable = 0).  Results are identical either way. */
MGM_API int mgm_use_compact(mgm_ctx *ctx, int enable);
/* One routine of the fractional step's reference-semantics multigrid on the
 * levels' p, source and residual (sweeps in data-parallel order):
 * relaxation (fractional_step_solver.h:168-196) or calculate_residuals
 * (:236-246) on `level`; restrict_residuals (:198-212) from `level` into
 * level + 1; prolongate_corrections (:214-234) from level + 1 into `level`. */
#define MGM_REF_RELAXATION 0
#define MGM_REF_RESIDUALS 1
#define MGM_REF_RESTRICT 2
#define MGM_REF_PROLONGATE 3
MGM_API int mgm_ref_routine(mgm_ctx *ctx, int level, int routine);
/* Replay captured CUDA graphs (default on) or launch every kernel one by one
 * (enable = 0).  With graphs on, mgm_step, mgm_run_steps, mgm_step_host and
 * the learned-start data collection run each fractional step in the FP64 /
 * FP32-IR modes as ONE graph launch (mgm_use_step_graph), and the other
 * solves replay each V-cycle from a captured graph.  Results are identical
 * either way. */
MGM_API int mgm_use_graphs(mgm_ctx *ctx, int enable);
/* V-cycle kernels after the first of a cycle or smoothing pass launched
 * with programmatic stream serialisation (enable = 1, default): a kernel's
 * CTAs may be scheduled while its predecessor's last CTAs finish, and wait
 * on the device for the predecessor's completion before touching memory, so
 * the launch latency between the ~100 kernels of a V-cycle overlaps.
 * enable = 0 launches them the ordinary way.  Results are identical. */
MGM_API int mgm_use_launch_chaining(mgm_ctx *ctx, int enable);
/* The levels below 65,536 rows (latency-bound: about 17 short kernels per
 * level per V-cycle) run as ONE cooperative launch per V-cycle, one CTA per
 * SM, a grid barrier between dependent passes (enable = 1, opt-in);
 * enable = 0 (default) launches every operation of those levels as its own
 * kernel, which measured faster on the 1M cavity (52 grid barriers per
 * V-cycle cost more than the launches they replace).  Results are
 * identical.  The barrier's wait is bounded: when it runs out the solve
 * returns MGM_ERR_TIMEOUT. */
MGM_API int mgm_use_fused_coarse(mgm_ctx *ctx, int enable);
/* 1 when the fused coarse V-cycle can run here (after mgm_setup: a CTA fits
 * on an SM and the driver accepts a cooperative kernel inside a conditional
 * graph node); 0: every level runs per-operation kernels whatever
 * mgm_use_fused_coarse says. */
MGM_API int mgm_fused_coarse_available(mgm_ctx *ctx, int *available);
/* Self-test of the bounded wait in the fused V-cycle's grid barrier: a
 * two-CTA cooperative launch in which one CTA never arrives, so the other's
 * wait runs out (under a second), records the timeout and returns; the
 * flags and the barrier are cleared after.  *status = MGM_ERR_TIMEOUT when
 * the bound worked (the context stays usable).  No reference counterpart. */
MGM_API int mgm_selftest_barrier_timeout(mgm_ctx *ctx, int *status);
/* With graphs on: the whole fractional step as one captured graph (enable =
 * 1, default) -- momentum, divergence, the Poisson solve with its restart and
 * Arnoldi loops as conditional WHILE nodes whose conditions device kernels
 * set, the velocity correction -- so that a step makes no host round trip;
 * or (enable = 0) the solve's loops driven from the host, which reads the
 * loop flags of the device-resident iteration state once per Arnoldi step
 * and replays each V-cycle from its graph.  The same kernels run in the same
 * order: results are identical.  The step graph is recaptured when dt, the
 * learned warm start or compatible right-hand sides change, and dropped by
 * every solver setting.  Profiling (mgm_profile_smoother) uses the
 * host-driven form, whose V-cycle graphs carry the timing events.  No
 * counterpart in the reference (fractional_step_solver.h:47-71 is one host
 * function). */
MGM_API int mgm_use_step_graph(mgm_ctx *ctx, int enable);
/* Counters of the Poisson solves of the last mgm_run_steps / mgm_step call
 * (read from the device-resident iteration state): Arnoldi steps (V-cycles),
 * restart-cycle starts (each computes a true residual), solves.  Any pointer
 * may be NULL.  No counterpart in the reference. */
MGM_API int mgm_solve_counters(mgm_ctx *ctx, long long *vcycles, long long *cycles, long long *solves);
/* Geometric mean, over the solves of the last run, of the relative residual
 * |b - A p0| / |b| each solve started from (p0 its initial guess,
 * mgm_set_initial_guess): what the guesses achieve before the first
 * V-cycle.  No reference counterpart. */
MGM_API int mgm_solve_start_residual(mgm_ctx *ctx, double *geo_mean);
/* FP32 compact path: on levels of at least 65,536 rows, stream the operator
 * tile by tile into shared memory with bulk asynchronous copies (enable = 1),
 * or read it with plain vector loads, four rows per thread (enable = 0, the
 * default, faster on B200).  Same results either way. */
MGM_API int mgm_use_tiled(mgm_ctx *ctx, int enable);
/* MGM_MODE_FP32_IR with a half-precision operator (enable = 1; default 0):
 * on levels of at least 65,536 rows the V-cycle's smoother and residual read
 * D^-1 A in FP16 packed with the int16 neighbour offsets (4 bytes per stencil
 * slot instead of 6), each row applied in difference form about its node so
 * that the row keeps its FP32 row sum; all sums stay FP32 and the FGMRES
 * refinement around the V-cycle stays FP64, so a solve still ends at the
 * relative residual set by mgm_set_solver.  A level whose scaled weights
 * leave FP16's range keeps its FP32 operator.  Results differ in rounding
 * from enable = 0 (a different preconditioner); the tile-streamed kernels of
 * mgm_use_tiled take precedence where enabled.  No counterpart in the
 * reference (its solver is FP64 throughout). */
MGM_API int mgm_use_half_operator(mgm_ctx *ctx, int enable);
/* MGM_MODE_FP64 / MGM_MODE_FP32_IR with compatible right-hand sides
 * (enable = 1; default 0).  lap_Poison (Laplacian interior rows, Neumann
 * boundary rows) is singular; the pinned solve (row 0 replaced by p[0] = 0)
 * otherwise puts the part of the source along the left null vector z into
 * row 0, a pressure spike at node 0 that a converged solve resolves and the
 * reference's non-converging cycles never do.  Enabled, each solve projects
 * the source to b - alpha w (w: 1 on interior rows, alpha = z.b / z.w) and
 * returns the pinned solution of that consistent system, which satisfies
 * every row of lap_Poison: p_b - alpha p_w, with alpha from the residuals of
 * the unpinned row-0 equation and p_w (the pinned solution for w) computed
 * once per set-up, here when the context is set up, else at the next solve.
 * The residual that mgm_last_solve and mgm_solve_poisson report is that of
 * the pinned solve for b, before the projection p_b - alpha p_w is applied
 * (p_w itself is solved to max(rel_tol, 1e-6)).
 * Applies to the fractional step, the TIMPLE p' solve and
 * mgm_solve_poisson.  No counterpart in the reference. */
MGM_API int mgm_set_compatible_rhs(mgm_ctx *ctx, int enable);
/* Statistics of the last Poisson solve: outer iterations (V-cycles) and the
 * true relative residual ||b - A p|| / ||b|| over rows != 0 (FP64). */
MGM_API int mgm_last_solve(mgm_ctx *ctx, int *iters, double *rel_res);

/* The fractional step's parts, on the device state
 * (fractional_step_solver.h:73-275).  mass_res may be NULL. */
MGM_API int mgm_intermediate_velocity(mgm_ctx *ctx);
MGM_API int mgm_mass_residual(mgm_ctx *ctx);
MGM_API int mgm_poisson(mgm_ctx *ctx, int mode);
MGM_API int mgm_update_velocity(mgm_ctx *ctx, double *mass_res);
/* sqrt(sum |u - u_old|^2 / n) of the last velocity update (fractional_step_solver.h:63-69). */
MGM_API int mgm_last_steady_error(mgm_ctx *ctx, double *steady_err);

/* Poisson solve of A p = b on level 0 (A = lap_Poison with row 0 replaced by
 * p[0] = 0), b given on the host (b[0] and boundary rows as given), p used as
 * the initial guess and returned.  The pinned row's rhs is forced to 0. */
MGM_API int mgm_solve_poisson(mgm_ctx *ctx, int mode, const double *b, double *p, int *iters, double *rel_res);

/* Runs nsteps fractional steps (as mgm_step) back to back and reports the
 * device time measured by CUDA events on the context's stream: total step
 * time, total Poisson-solve time and V-cycles used.  Any output may be NULL.
 * (No reference counterpart: measurement hook for fractional_step_explicit loops.) */
MGM_API int mgm_run_steps(mgm_ctx *ctx, int mode, int nsteps, double *step_ms, double *poisson_ms,
                          long long *vcycles, double *steady_err);

/* One fractional step with host buffers, the shape of the reference's time
 * loop (mg_NS_solver.c:68-91: step, then `acc update host(field[0])`):
 * uploads the given level-0 velocity components (NULL = keep the device
 * copy), steps, and downloads u, v, w, p into the given buffers (NULL = skip).
 * Use mgm_host_alloc for page-locked buffers. */
MGM_API int mgm_step_host(mgm_ctx *ctx, int mode, const double *u_in, const double *v_in, const double *w_in,
                          double *u_out, double *v_out, double *w_out, double *p_out, double *steady_err);
MGM_API void *mgm_host_alloc(size_t bytes);
MGM_API void mgm_host_free(void *ptr);

/* Per-launch device timing of the level-0 smoother kernel (the dominant
 * kernel of the FP32-in-FP64 solve).  bytes_per_launch is its algorithmic
 * traffic (operator, index and vector bytes, each counted once). */
MGM_API int mgm_profile_smoother(mgm_ctx *ctx, int enable);
MGM_API int mgm_profile_read(mgm_ctx *ctx, double *ms_total, long long *launches, long long *bytes_per_launch);

/* ------------------------------------------------------------------ */
/* Learned warm start (no counterpart in the reference)                */
/* ------------------------------------------------------------------ */
/* The initial guess of each fractional step's Poisson solve (FP64 and
 * FP32-IR modes).  By default (flags 0) the solve starts from the previous
 * step's pressure, as the reference's p does.  MGM_GUESS_EXTRAPOLATE adds the
 * direction p_prev - p_prev2 (the last pressure increment; none right after
 * mgm_apply_bc), MGM_GUESS_LEARNED the network's predicted increment
 * (mgm_set_warm_start); the solve starts from p_prev + sum_i c_i d_i with
 * the coefficients that minimise the FP64 residual |b - A p|_2 (a minimal-
 * residual step over the directions: never a larger starting residual than
 * p_prev), then iterates to the same tolerance.  Guesses apply to mgm_step,
 * mgm_run_steps, mgm_step_host and mgm_mpnn_collect; they need max_iters >= 4
 * (the directions are staged in the Krylov basis).  No counterpart in the
 * reference. */
#define MGM_GUESS_EXTRAPOLATE 1
#define MGM_GUESS_LEARNED 2
MGM_API int mgm_set_initial_guess(mgm_ctx *ctx, int flags);
/* A 4-layer message-passing network (hidden width 64, BF16 weights and
 * activations, FP32 accumulation) on the level-0 stencil graph predicts the
 * part of a Poisson solve's pressure increment that extrapolating the last
 * increment misses, from (b, previous p, the last increment p_prev - p_prev2,
 * coordinates).  With the warm start on
 * (mgm_set_warm_start: the MGM_GUESS_LEARNED bit of mgm_set_initial_guess)
 * each step's solve starts from the minimal-residual combination of the
 * prediction (and, with MGM_GUESS_EXTRAPOLATE, the last increment); the
 * V-cycle-preconditioned FGMRES then runs to the same tolerance as without
 * it.  mgm_mpnn_init allocates it (seeded weights) and a dataset ring of
 * dataset_capacity samples (4 n floats each); mgm_mpnn_collect runs time
 * steps with a solver mode and records (b, p_prev, dp = p_prev - p_prev2,
 * (p_new - p_prev) - dp: the part of the new increment the extrapolation
 * misses, which the network learns), each normalised by its RMS; mgm_mpnn_train runs Adam on a
 * range of samples (losses[it] per iteration, may be NULL); mgm_mpnn_eval
 * returns the mean loss on a range.  Params: mgm_mpnn_num_params() floats. */
MGM_API int mgm_mpnn_init(mgm_ctx *ctx, unsigned long long seed, int dataset_capacity);
MGM_API int mgm_mpnn_num_params(void);
MGM_API int mgm_mpnn_params(mgm_ctx *ctx, float *get, const float *set);
MGM_API int mgm_mpnn_loss_grad(mgm_ctx *ctx, const float *b_hat, const float *p_hat, const float *dp_hat,
                               const float *target, double *loss, float *grads, float *prediction);
/* The inference pass a step runs (the decoder fused into the last layer,
 * no activations kept) on normalised host inputs; prediction: n floats. */
MGM_API int mgm_mpnn_predict(mgm_ctx *ctx, const float *b_hat, const float *p_hat, const float *dp_hat,
                             float *prediction);
MGM_API int mgm_mpnn_collect(mgm_ctx *ctx, int mode, int nsteps);
MGM_API int mgm_mpnn_dataset_size(mgm_ctx *ctx, int *count);
MGM_API int mgm_mpnn_train(mgm_ctx *ctx, int first, int count, int iters, float lr, unsigned long long seed,
                           double *losses);
MGM_API int mgm_mpnn_eval(mgm_ctx *ctx, int first, int count, double *mean_loss);
/* Training loss w_mse * mean (y - t)^2 + w_res * |A (t - y)|^2 / |A t|^2,
 * t the normalised increment, A the pinned Poisson operator: the second term
 * is the starting residual the prediction leaves (default 1, 0). */
MGM_API int mgm_mpnn_set_loss(mgm_ctx *ctx, float w_mse, float w_res);
MGM_API int mgm_set_warm_start(mgm_ctx *ctx, int enable);
/* Fine-level Chebyshev steps applied to the learned direction before the
 * minimal-residual step (default 3; 0 = use the raw prediction), and the
 * coefficient the last step's solve took along it. */
MGM_API int mgm_set_warm_smoothing(mgm_ctx *ctx, int steps);
MGM_API int mgm_last_learned_alpha(mgm_ctx *ctx, double *alpha);

/* Synchronises the context's stream. */
MGM_API int mgm_sync(mgm_ctx *ctx);

/* ------------------------------------------------------------------ */
/* Batched hierarchies: per-node stencil sizes, one-launch weight      */
/* assembly, many right-hand sides through one V-cycle.               */
/* No counterpart in the reference, which has one stencil size per    */
/* level (structures.h:15-78, mesh_functions.h:131-170) and one       */
/* right-hand side per solve (fractional_step_solver.h:150-166).      */
/* ------------------------------------------------------------------ */
typedef struct mgm_batch mgm_batch;
MGM_API mgm_batch *mgm_batch_create(int dim, int phs_degree, int num_levels);
MGM_API void mgm_batch_destroy(mgm_batch *b);
/* Level input as for mgm_set_level (boundary nodes first, no corners), with
 * the stencil size of every node: k_per_node[i] nearest nodes (self first;
 * boundary node: itself then k-1 interior nodes, kdtree_functions.h:141-149). */
MGM_API int mgm_batch_set_level(mgm_batch *b, int lev, int n, int nb, const double *x, const double *y,
                                const double *z, const double *nx, const double *ny, const double *nz,
                                const unsigned char *btag, int poly_degree, const int *k_per_node);
#define MGM_BATCH_AUTOTUNE 1 /* time candidate team widths / CTA budgets before the launch */
/* kNN lists, breadth-first reorder, normals, nearest points, then every
 * derivative row (rbf.h:401-421), restriction row and prolongation row
 * (mesh_functions.h:533-670) of every level in ONE persistent launch, then the
 * solver set-up (pinned operators, smoother bounds, coarsest inverse). */
MGM_API int mgm_batch_setup(mgm_batch *b, int flags);
/* The weight launch: its device time, the autotuner's time, systems, tiles,
 * shared memory per CTA and resident CTAs per SM. */
MGM_API int mgm_batch_weights_report(mgm_batch *b, double *weights_ms, double *tuning_ms, long long *systems,
                                     int *tiles, int *smem_bytes, int *ctas_per_sm);
/* Size classes (largest system order first): order N = k + np, systems,
 * threads per system chosen, measured microseconds per system (0 untuned). */
MGM_API int mgm_batch_num_classes(mgm_batch *b, int *count);
MGM_API int mgm_batch_class(mgm_batch *b, int idx, int *order, long long *systems, int *team_threads,
                            double *us_per_system);
MGM_API int mgm_batch_level_size(mgm_batch *b, int lev, int *n, int *nb, long long *nnz, long long *r_nnz,
                                 long long *p_nnz);
/* Level data after the reorder (CSR: row i = col[row_ptr[i] .. row_ptr[i+1])).
 * Any output may be NULL. */
MGM_API int mgm_batch_get_level(mgm_batch *b, int lev, double *x, double *y, double *z, double *nx, double *ny,
                                double *nz, unsigned char *btag, int *k_per_node, int *row_ptr, int *col,
                                double *Dx, double *Dy, double *Dz, double *lap, double *lapP);
/* Restriction into level lev (row i interpolates level lev-1 at node i; rows
 * of boundary nodes and node 0 are empty) and prolongation into level lev
 * (from level lev+1, every row).  Any output may be NULL. */
MGM_API int mgm_batch_get_transfer(mgm_batch *b, int lev, int *rpts, int *ppts, int *r_ptr, int *r_col,
                                   double *r_w, int *p_ptr, int *p_col, double *p_w);
/* rel_tol, Krylov restart length (<= 32), Chebyshev degree and ratio. */
MGM_API int mgm_batch_set_solver(mgm_batch *b, double rel_tol, int restart, int cheb_degree, double cheb_ratio);
/* Solves the pinned Poisson system (row 0 -> p[0] = 0) for nrhs <= 64
 * right-hand sides at once: rhs and sol are host arrays [nrhs][n0] in the
 * reordered node order; rel_res[nrhs].  mode: MGM_MODE_FP64 or
 * MGM_MODE_FP32_IR.  solve_ms: device time with the right-hand sides in HBM. */
MGM_API int mgm_batch_solve(mgm_batch *b, int mode, int nrhs, const double *rhs, double *sol, int *vcycles,
                            double *rel_res, double *solve_ms);

#ifdef __cplusplus
}
#endif
#endif
