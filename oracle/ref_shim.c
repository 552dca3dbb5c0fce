/*
 * ref_shim.c -- TEST INFRASTRUCTURE ONLY (never shipped, never on the product path).
 *
 * Compiles the reference solver's own, unmodified C headers (Multigrid_meshless
 * header_files/*.h and init/init_{LDC,TC}.c, included from the reference tree at
 * build time, see oracle/Makefile) into oracle/_ref/libref.so and exposes a flat,
 * ctypes-friendly handle so that the tests can run the reference's functions on
 * the project's synthetic clouds:
 *
 *   find_cloud_index                  kdtree_functions.h:113-151
 *   rcm_reordering_with_boundarynodes mesh_functions.h:774-872
 *   correct_normal_directions         mesh_functions.h:478-527
 *   calculate_avg_dx                  mesh_functions.h:895-910
 *   create_prolongation_and_restriction_matrices  mesh_functions.h:874-893
 *   create_derivative_matrices        rbf.h:401-421
 *   calculate_dt                      general_functions.h:34-41
 *   fractional_step_explicit & callees  fractional_step_solver.h:47-275
 *   time_implicit_solver & callees    timple_solver.h:40-410 (built with
 *                                     -DMGM_REF_TIMPLE into _ref/libref_timple.so)
 *   read_PointStructure               mesh_functions.h:172-476 (the Gmsh reader;
 *                                     ref_read_mesh)
 *   the heat-conduction program's routines  heat_conduction.h:24-113 and
 *                                     init/init_heat_conduction.c:14-67 (built
 *                                     with -DMGM_REF_HEAT into _ref/libref_heat.so)
 *
 * The level set-up mirrors read_complete_mesh_data (mesh_functions.h:914-928)
 * with the mesh reader replaced by arrays handed in by the caller (boundary
 * nodes first, no corner nodes -- the state read_PointStructure leaves behind,
 * mesh_functions.h:434-473).  free_PointStructure is never called: it frees rows
 * that were never allocated (structures.h:174-209).
 */
#include <stdio.h>
#include <string.h>
#if defined(MGM_REF_HEAT)
/* _ref/libref_heat.so: the same handle over the heat-conduction program's
 * routines (heat_conduction.h:24-113, init/init_heat_conduction.c:14-67) */
#include "header_files/heat_conduction.h"
#include "init/init_heat_conduction.c"
#else
#ifdef MGM_REF_TIMPLE
/* _ref/libref_timple.so: the same handle over the reference's time-implicit
 * (TIMPLE) solver, timple_solver.h:40-410, the default of mg_NS_solver.c */
#include "header_files/timple_solver.h"
#else
#include "header_files/fractional_step_solver.h"
#endif
#include "init/init_LDC.c"
#undef INIT_C
#define initial_conditions tc_initial_conditions
#define boundary_conditions tc_boundary_conditions
#include "init/init_TC.c"
#undef initial_conditions
#undef boundary_conditions
#endif

static PointStructure *g_ps = NULL;
static FieldVariables *g_field = NULL;
static int g_levels = 0;

int ref_begin(int dim, int phs_degree, int num_levels)
{
    memset(&parameters, 0, sizeof(parameters));
    parameters.dimension = (short)dim;
    parameters.phs_degree = (short)phs_degree;
    parameters.num_levels = (short)num_levels;
    /* Leaked on purpose between cases (see header): tests create few handles. */
    g_ps = (PointStructure *)calloc((size_t)num_levels, sizeof(PointStructure));
    g_field = NULL;
    g_levels = num_levels;
    return g_ps ? 0 : -1;
}

/* Mirrors the tail of read_flow_parameters (mesh_functions.h:97-99). */
void ref_set_flow(double courant, double Re, float omega, int num_vcycles, int num_relax)
{
    parameters.courant_number = courant;
    parameters.Re = Re;
    parameters.omega = omega;
    parameters.num_vcycles = (short)num_vcycles;
    parameters.num_relax = (short)num_relax;
    parameters.rho = 1;
    parameters.mu = parameters.rho / parameters.Re;
    parameters.nu = parameters.mu / parameters.rho;
}

int ref_set_level(int lev, int n, int nb, const double *x, const double *y, const double *z,
                  const double *nx, const double *ny, const double *nz,
                  const unsigned char *btag, int poly_degree, int k, double d_avg)
{
    PointStructure *p = &g_ps[lev];
    p->poly_degree = (short)poly_degree;
    calculate_parameters(p);
    p->num_cloud_points = (short)k; /* k set directly (structures.h:20 only allows short multiples) */
    AllocateMemoryPointStructure(p, n);
    for (int i = 0; i < n; i++) {
        p->x[i] = x[i]; p->y[i] = y[i]; p->z[i] = z[i];
        p->x_normal[i] = nx[i]; p->y_normal[i] = ny[i]; p->z_normal[i] = nz[i];
        p->boundary_tag[i] = btag[i] != 0;
        p->corner_tag[i] = false;
        p->point_index[i] = i;
    }
    p->num_boundary_nodes = nb;
    p->num_corners = 0;
    p->d_avg = d_avg;
    return 0;
}

void ref_clouds(int lev) { find_cloud_index(&g_ps[lev]); }
void ref_rcm(int lev) { rcm_reordering_with_boundarynodes(&g_ps[lev]); }
void ref_normals(int lev) { correct_normal_directions(&g_ps[lev]); }
double ref_avg_dx(int lev) { calculate_avg_dx(&g_ps[lev]); return g_ps[lev].d_avg; }
void ref_set_davg(int lev, double d) { g_ps[lev].d_avg = d; }
void ref_rp(void) { create_prolongation_and_restriction_matrices(g_ps, (short)g_levels); }
void ref_derivatives(int lev) { create_derivative_matrices(&g_ps[lev]); }

int ref_num_poly_terms(int lev) { return g_ps[lev].num_poly_terms; }

void ref_get_geometry(int lev, double *x, double *y, double *z, double *nx, double *ny, double *nz,
                      unsigned char *btag, int *cloud)
{
    PointStructure *p = &g_ps[lev];
    int k = p->num_cloud_points;
    for (int i = 0; i < p->num_nodes; i++) {
        x[i] = p->x[i]; y[i] = p->y[i]; z[i] = p->z[i];
        nx[i] = p->x_normal[i]; ny[i] = p->y_normal[i]; nz[i] = p->z_normal[i];
        btag[i] = p->boundary_tag[i] ? 1 : 0;
        for (int j = 0; j < k; j++) cloud[(size_t)i * k + j] = p->cloud_index[i][j];
    }
}

/* Operators as row-major [n][k]; Dz only read when dim == 3. */
void ref_get_ops(int lev, double *Dx, double *Dy, double *Dz, double *lap, double *lapP)
{
    PointStructure *p = &g_ps[lev];
    int k = p->num_cloud_points;
    for (int i = 0; i < p->num_nodes; i++)
        for (int j = 0; j < k; j++) {
            size_t o = (size_t)i * k + j;
            Dx[o] = p->Dx[i][j]; Dy[o] = p->Dy[i][j]; lap[o] = p->lap[i][j]; lapP[o] = p->lap_Poison[i][j];
            if (parameters.dimension == 3) Dz[o] = p->Dz[i][j];
        }
}

/* restriction_points / prolongation_points of a level, and its restr_mat
 * (width k of the finer level; absent on level 0) / prol_mat (width k of the
 * coarser level; absent on the coarsest level). */
void ref_get_transfer(int lev, int *rpts, int *ppts, double *restr, double *prol)
{
    PointStructure *p = &g_ps[lev];
    for (int i = 0; i < p->num_nodes; i++) { rpts[i] = p->restriction_points[i]; ppts[i] = p->prolongation_points[i]; }
    if (lev > 0 && restr) {
        int kf = g_ps[lev - 1].num_cloud_points;
        for (int i = 0; i < p->num_nodes; i++)
            for (int j = 0; j < kf; j++) restr[(size_t)i * kf + j] = p->restr_mat[i][j];
    }
    if (lev < g_levels - 1 && prol) {
        int kc = g_ps[lev + 1].num_cloud_points;
        for (int i = 0; i < p->num_nodes; i++)
            for (int j = 0; j < kc; j++) prol[(size_t)i * kc + j] = p->prol_mat[i][j];
    }
}

/* Hands a level's clouds and derivative operators (row-major [n][k], built
 * elsewhere -- e.g. by the restatement, whose set-up is pinned bit for bit to
 * find_cloud_index + create_derivative_matrices) to the reference's
 * structures, allocated row by row as kdtree_functions.h:115-118 and
 * rbf.h:401-421 allocate them.  Dz is read only when dim == 3. */
void ref_load_ops(int lev, const int *cloud, const double *Dx, const double *Dy, const double *Dz, const double *lap,
                  const double *lapP)
{
    PointStructure *p = &g_ps[lev];
    const int n = p->num_nodes, k = p->num_cloud_points;
    const int d3 = parameters.dimension == 3;
    p->cloud_index = (int **)malloc(sizeof(int *) * (size_t)n);
    for (int i = 0; i < n; i++) {
        p->cloud_index[i] = (int *)malloc(sizeof(int) * (size_t)k);
        memcpy(p->cloud_index[i], cloud + (size_t)i * k, sizeof(int) * (size_t)k);
    }
    /* one matrix after the other, rows consecutively, in create_derivative_matrices' order */
    double ***ops[5] = {&p->Dx, &p->Dy, &p->lap, &p->Dz, &p->lap_Poison};
    const double *src[5] = {Dx, Dy, lap, Dz, lapP};
    for (int o = 0; o < 5; o++) {
        if (o == 3 && !d3) { p->Dz = NULL; continue; }
        double **m = (double **)malloc(sizeof(double *) * (size_t)n);
        for (int i = 0; i < n; i++) {
            m[i] = (double *)malloc(sizeof(double) * (size_t)k);
            memcpy(m[i], src[o] + (size_t)i * k, sizeof(double) * (size_t)k);
        }
        *ops[o] = m;
    }
}

/* The transfer data of a level, as create_prolongation_and_restriction_matrices
 * (mesh_functions.h:874-893) leaves it: restriction / prolongation points [n],
 * restr_mat [n][k of the finer level] (levels > 0), prol_mat [n][k of the
 * coarser level] (all but the coarsest), allocated row by row. */
void ref_load_transfer(int lev, const int *rpts, const int *ppts, const double *restr, const double *prol)
{
    PointStructure *p = &g_ps[lev];
    const int n = p->num_nodes;
    p->restriction_points = (int *)malloc(sizeof(int) * (size_t)n);
    p->prolongation_points = (int *)malloc(sizeof(int) * (size_t)n);
    memcpy(p->restriction_points, rpts, sizeof(int) * (size_t)n);
    memcpy(p->prolongation_points, ppts, sizeof(int) * (size_t)n);
    if (lev > 0 && restr) {
        const int kf = g_ps[lev - 1].num_cloud_points;
        p->restr_mat = (double **)malloc(sizeof(double *) * (size_t)n);
        for (int i = 0; i < n; i++) {
            p->restr_mat[i] = (double *)malloc(sizeof(double) * (size_t)kf);
            memcpy(p->restr_mat[i], restr + (size_t)i * kf, sizeof(double) * (size_t)kf);
        }
    }
    if (lev < g_levels - 1 && prol) {
        const int kc = g_ps[lev + 1].num_cloud_points;
        p->prol_mat = (double **)malloc(sizeof(double *) * (size_t)n);
        for (int i = 0; i < n; i++) {
            p->prol_mat[i] = (double *)malloc(sizeof(double) * (size_t)kc);
            memcpy(p->prol_mat[i], prol + (size_t)i * kc, sizeof(double) * (size_t)kc);
        }
    }
}

/* ---- fields and the fractional step ---------------------------------- */
void ref_fields_alloc(void) { AllocateMemoryFieldVariables(&g_field, g_ps, g_levels); }

#ifndef MGM_REF_HEAT
/* kind 0: lid-driven cavity (init_LDC.c), kind 1: Taylor-Couette (init_TC.c).
 * Applied to level 0 only, as mg_NS_solver.c:49-50 does. */
void ref_bc(int kind)
{
    if (kind == 0) { initial_conditions(g_ps, g_field, 1); boundary_conditions(g_ps, g_field, 1); }
    else { tc_initial_conditions(g_ps, g_field, 1); tc_boundary_conditions(g_ps, g_field, 1); }
}
#endif

double ref_dt(void) { parameters.dt = calculate_dt(&g_ps[0]); return parameters.dt; }
void ref_set_dt(double dt) { parameters.dt = dt; }

static double *field_ptr(int lev, int which)
{
    FieldVariables *f = &g_field[lev];
    switch (which) {
    case 0: return f->u; case 1: return f->v; case 2: return f->w; case 3: return f->p;
    case 4: return f->u_new; case 5: return f->v_new; case 6: return f->w_new;
    case 7: return f->u_old; case 8: return f->v_old; case 9: return f->w_old;
    case 10: return f->res; case 11: return f->source; case 12: return f->dpdn;
    case 13: return f->dpdx; case 14: return f->dpdy; case 15: return f->dpdz;
    case 16: return f->p_old; case 17: return f->pprime;
    }
    return NULL;
}
void ref_field_get(int lev, int which, double *out) { memcpy(out, field_ptr(lev, which), sizeof(double) * g_ps[lev].num_nodes); }
void ref_field_set(int lev, int which, const double *in) { memcpy(field_ptr(lev, which), in, sizeof(double) * g_ps[lev].num_nodes); }

#if defined(MGM_REF_HEAT)
/* mg_heat_conduction.c:47-48: initial and boundary conditions of wave number k */
void ref_heat_init(int wave)
{
    initial_conditions(g_ps, g_field, g_levels, wave);
    boundary_conditions(g_ps, g_field, g_levels, wave);
}
/* one pass of the time loop of mg_heat_conduction.c:55-77 (the program's own
 * V-cycle after set_boundary_rhs, num_vcycles times); returns its
 * steady_state_error, the sum of squared changes of p on level 0 */
double ref_heat_step(int wave)
{
    const int n = g_ps[0].num_nodes, nl = g_levels;
    double *temp = (double *)malloc(sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) temp[i] = g_field[0].p[i];
    for (int icycle = 0; icycle < parameters.num_vcycles; icycle++) {
        set_boundary_rhs(&g_ps[0], g_field, nl, wave);
        for (int ilev = 0; ilev < nl; ilev++) {
            relaxation(&g_ps[ilev], &g_field[ilev]);
            calculate_residuals(&g_ps[ilev], &g_field[ilev]);
            if (ilev != nl - 1) restrict_residuals(&g_ps[ilev], &g_ps[ilev + 1], &g_field[ilev], &g_field[ilev + 1]);
        }
        for (int ilev = nl - 1; ilev > 0; ilev--) {
            prolongate_corrections(&g_ps[ilev - 1], &g_ps[ilev], &g_field[ilev - 1], &g_field[ilev]);
            if (ilev != 1) relaxation(&g_ps[ilev - 1], &g_field[ilev - 1]);
        }
    }
    double e = 0.0;
    for (int i = 0; i < n; i++) e += (temp[i] - g_field[0].p[i]) * (temp[i] - g_field[0].p[i]);
    free(temp);
    return e;
}
#elif defined(MGM_REF_TIMPLE)
/* TIMPLE parameters (read_flow_parameters, mesh_functions.h:82-91).  The
 * reference never sets FieldVariables.rho, which update_boundary_pressure
 * (timple_solver.h:365) reads; it is defined here as parameters.rho. */
void ref_timple_params(int iter_timple, int iter_momentum, double facRe, double facdt)
{
    parameters.iter_timple = (short)iter_timple;
    parameters.iter_momentum = (short)iter_momentum;
    parameters.facRe = facRe;
    parameters.facdt = facdt;
    for (int l = 0; l < g_levels; l++) { g_field[l].rho = parameters.rho; g_field[l].mu = parameters.mu; }
}
double ref_timple_step(void) { return time_implicit_solver(g_ps, g_field); }
void ref_timple_momentum(void) { calculate_intermediate_velocity_implicit(&g_ps[0], &g_field[0]); }
void ref_timple_mass(void) { calculate_mass_residual_implicit(&g_ps[0], &g_field[0]); }
void ref_timple_update_velocity(void) { update_velocity_implicit(&g_ps[0], &g_field[0]); }
void ref_timple_boundary_pressure(void) { update_boundary_pressure(&g_ps[0], &g_field[0]); }
#else
double ref_step(void) { return fractional_step_explicit(g_ps, g_field); }
void ref_intermediate_velocity(void) { calculate_intermediate_velocity(&g_ps[0], &g_field[0]); }
void ref_mass_residual(void) { calculate_mass_residual(&g_ps[0], &g_field[0]); }
void ref_boundary_dpdn(void) { calculate_boundary_dpdn(&g_ps[0], &g_field[0]); }
void ref_update_velocity(void) { update_velocity(&g_ps[0], &g_field[0]); }
#endif
#ifndef MGM_REF_HEAT
void ref_multigrid(void) { multigrid_Poisson_solver(g_ps, g_field); }
#endif
void ref_relaxation(int lev) { relaxation(&g_ps[lev], &g_field[lev]); }
void ref_residuals(int lev) { calculate_residuals(&g_ps[lev], &g_field[lev]); }
void ref_restrict(int lev) { restrict_residuals(&g_ps[lev], &g_ps[lev + 1], &g_field[lev], &g_field[lev + 1]); }
void ref_prolongate(int lev) { prolongate_corrections(&g_ps[lev], &g_ps[lev + 1], &g_field[lev], &g_field[lev + 1]); }
void ref_spmv(int lev, int op, const double *f, double *out)
{
    PointStructure *p = &g_ps[lev];
    double **D = op == 0 ? p->Dx : op == 1 ? p->Dy : op == 2 ? p->Dz : op == 3 ? p->lap : p->lap_Poison;
    multiply_sparse_matrix_vector_gpu(D, (double *)f, out, p->cloud_index, p->num_nodes, p->num_cloud_points);
}

/* read_PointStructure (mesh_functions.h:172-476) on a Gmsh file: returns the
 * node count after corner removal; with cap >= that count the arrays are
 * filled.  The path must be shorter than PointStructure.mesh_filename (50). */
int ref_read_mesh(const char *path, int dim, int cap, double *x, double *y, double *z, double *nx, double *ny,
                  double *nz, unsigned char *btag, unsigned char *corner, int *nb, int *num_elem, double *d_avg)
{
    PointStructure p;
    memset(&p, 0, sizeof(p));
    if (strlen(path) >= sizeof(p.mesh_filename)) return -1;
    strcpy(p.mesh_filename, path);
    parameters.dimension = (short)dim;
    read_PointStructure(&p);
    const int n = p.num_nodes;
    *nb = p.num_boundary_nodes;
    *num_elem = p.num_elem;
    *d_avg = p.d_avg;
    if (cap >= n) {
        for (int i = 0; i < n; i++) {
            x[i] = p.x[i]; y[i] = p.y[i]; z[i] = p.z[i];
            nx[i] = p.x_normal[i]; ny[i] = p.y_normal[i]; nz[i] = p.z_normal[i];
            btag[i] = p.boundary_tag[i]; corner[i] = p.corner_tag[i];
        }
    }
    return n;
}

/* write_processed_grid_data (write_functions.h:186-201) of a level into the
 * working directory, and write_test_files (:124-184) with prefix `folder` */
void ref_write_grid(int lev) { write_processed_grid_data(&g_ps[lev], lev); }
void ref_write_test_files(double *f, double *fx, double *fy, double *fz, double *lapf, double *fxx, double *fyy,
                          double *fzz, int n, char *folder)
{
    write_test_files(f, fx, fy, fz, lapf, fxx, fyy, fzz, n, folder);
}

/* matrixInverse_Gauss_Jordan (mat_lib.h:423-491) on a row-major N x N matrix */
void ref_gauss_jordan(int N, const double *A, double *Ainv)
{
    double **a = (double **)malloc(sizeof(double *) * (size_t)N), **b = (double **)malloc(sizeof(double *) * (size_t)N);
    for (int i = 0; i < N; i++) {
        a[i] = (double *)malloc(sizeof(double) * (size_t)N);
        b[i] = (double *)malloc(sizeof(double) * (size_t)N);
        for (int j = 0; j < N; j++) a[i][j] = A[(size_t)i * N + j];
    }
    matrixInverse_Gauss_Jordan(a, b, N);
    for (int i = 0; i < N; i++) {
        for (int j = 0; j < N; j++) Ainv[(size_t)i * N + j] = b[i][j];
        free(a[i]);
        free(b[i]);
    }
    free(a);
    free(b);
}
