/*
 * legacy_driver.c -- a program written against the reference's call surface
 * (the flow of mg_NS_solver.c:17-103 with the mesh reader replaced by a node
 * file), linked against libmgm.so through include/mgm_reference.h.
 *
 *   legacy_driver <input.bin> <output_dir> [timple|routines]
 *   legacy_driver --gmsh <flow_parameters.csv> <grid_filenames.csv> <output_dir>
 *
 * The --gmsh form is mg_NS_solver.c:17-45 as written: read_flow_parameters,
 * read_grid_filenames, read_complete_mesh_data on Gmsh files (the reference's
 * own reader semantics, mesh_functions.h:172-476, 914-928), then
 * num_time_steps fractional steps on the lid-driven cavity.
 *
 * With "timple" the time loop is the reference main's default,
 * time_implicit_solver (timple_solver.h:40-70), on the Taylor-Couette
 * conditions of init_TC.c (iter_timple = iter_momentum = 2, facRe = facdt = 1);
 * otherwise fractional_step_explicit on the lid-driven cavity (init_LDC.c).
 * With "routines" the operators come from create_full_gradx/grady/gradz/
 * laplacian_matrix and create_laplacian_for_Poisson, and each step calls the
 * fractional step's parts and multigrid routines one by one (the cycle of
 * multigrid_Poisson_solver, fractional_step_solver.h:150-166, written out);
 * it also writes the inverse of a small matrix by matrixInverse_Gauss_Jordan.
 *
 * input.bin: int32 nl, dim, phs, poly, multiplier, nsteps, num_vcycles,
 *            num_relax, mode; double Re, courant, omega; per level: int32 n,
 *            nb; double x[n], y[n], z[n], nx[n], ny[n], nz[n]; uint8 btag[n].
 * Writes raw arrays into output_dir (read back by tests/test_gpu_legacy.py).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mgm_reference.h"

static void rd(void *p, size_t sz, size_t n, FILE *f)
{
    if (fread(p, sz, n, f) != n) { fprintf(stderr, "short read\n"); exit(2); }
}

static void wr(const char *dir, const char *name, const void *p, size_t bytes)
{
    char path[512];
    snprintf(path, sizeof(path), "%s/%s", dir, name);
    FILE *f = fopen(path, "wb");
    if (!f || fwrite(p, 1, bytes, f) != bytes) { fprintf(stderr, "write %s failed\n", path); exit(3); }
    fclose(f);
}

static void wr_rows_d(const char *dir, const char *name, double **rows, int n, int k)
{
    double *flat = malloc(sizeof(double) * (size_t)n * k);
    for (int i = 0; i < n; i++) memcpy(flat + (size_t)i * k, rows[i], sizeof(double) * k);
    wr(dir, name, flat, sizeof(double) * (size_t)n * k);
    free(flat);
}

static void wr_rows_i(const char *dir, const char *name, int **rows, int n, int k)
{
    int *flat = malloc(sizeof(int) * (size_t)n * k);
    for (int i = 0; i < n; i++) memcpy(flat + (size_t)i * k, rows[i], sizeof(int) * k);
    wr(dir, name, flat, sizeof(int) * (size_t)n * k);
    free(flat);
}

static int read_bin(const char *path, PointStructure **out_ps, int *out_nsteps);
static int run(PointStructure *ps, int nl, int nsteps, int kind, const char *out);
static void step_by_routines(PointStructure *ps, FieldVariables *field, int nl);

int main(int argc, char **argv)
{
    if (argc < 3) { fprintf(stderr, "usage: legacy_driver input.bin outdir [timple|routines]\n"); return 1; }
    const int gmsh = argc >= 5 && strcmp(argv[1], "--gmsh") == 0;
    const int timple = !gmsh && argc > 3 && strcmp(argv[3], "timple") == 0;
    const int routines = !gmsh && argc > 3 && strcmp(argv[3], "routines") == 0;
    const char *out = gmsh ? argv[4] : argv[2];
    PointStructure *ps = NULL;
    int nl = 0, nsteps = 0;
    if (gmsh) {
        /* mg_NS_solver.c:21-45 */
        short num_levels = 0;
        read_flow_parameters(argv[2]);
        read_grid_filenames(&ps, argv[3], &num_levels);
        parameters.num_levels = num_levels;
        read_complete_mesh_data(ps, num_levels);
        nl = num_levels;
        nsteps = parameters.num_time_steps;
    } else {
        nl = read_bin(argv[1], &ps, &nsteps);
    }
    for (int l = 0; l < nl; l++) {
        if (!routines) {
            create_derivative_matrices(&ps[l]);
            continue;
        }
        create_full_gradx_matrix(&ps[l]);
        create_full_grady_matrix(&ps[l]);
        if (parameters.dimension == 3) create_full_gradz_matrix(&ps[l]);
        create_full_laplacian_matrix(&ps[l]);
        create_laplacian_for_Poisson(&ps[l]);
    }
    if (routines) {
        /* a 5 x 5 matrix with a zero first pivot */
        double a[5][5] = {{0, 2, 1, 0, 3}, {2, 0, 4, 1, 0}, {1, 4, 0, 2, 1}, {0, 1, 2, 5, 1}, {3, 0, 1, 1, 6}};
        double *ar[5], *br[5], inv[25];
        for (int i = 0; i < 5; i++) { ar[i] = a[i]; br[i] = inv + 5 * i; }
        matrixInverse_Gauss_Jordan(ar, br, 5);
        wr(out, "gj_inverse", inv, sizeof(inv));
    }
    return run(ps, nl, nsteps, timple ? 1 : (routines ? 2 : 0), out);
}

/* fractional_step_explicit (fractional_step_solver.h:47-71) through its parts,
 * the multigrid written out with the per-level routines */
static void step_by_routines(PointStructure *ps, FieldVariables *field, int nl)
{
    calculate_intermediate_velocity(&ps[0], &field[0]);
    calculate_mass_residual(&ps[0], &field[0]);
    calculate_boundary_dpdn(&ps[0], &field[0]);
    for (int cyc = 0; cyc < parameters.num_vcycles; cyc++) {
        for (int l = 0; l < nl; l++) {
            relaxation(&ps[l], &field[l]);
            calculate_residuals(&ps[l], &field[l]);
            if (l != nl - 1) restrict_residuals(&ps[l], &ps[l + 1], &field[l], &field[l + 1]);
        }
        for (int l = nl - 1; l > 0; l--) {
            prolongate_corrections(&ps[l - 1], &ps[l], &field[l - 1], &field[l]);
            if (l != 1) relaxation(&ps[l - 1], &field[l - 1]);
        }
    }
    update_velocity(&ps[0], &field[0]);
}

/* nodes from input.bin, then the steps of read_complete_mesh_data after the reader */
static int read_bin(const char *path, PointStructure **out_ps, int *out_nsteps)
{
    FILE *f = fopen(path, "rb");
    if (!f) { fprintf(stderr, "cannot open %s\n", path); exit(1); }
    int hdr[9];
    double flow[3];
    rd(hdr, sizeof(int), 9, f);
    rd(flow, sizeof(double), 3, f);
    const int nl = hdr[0];
    *out_nsteps = hdr[5];
    memset(&parameters, 0, sizeof(parameters));
    parameters.dimension = (short)hdr[1];
    parameters.phs_degree = (short)hdr[2];
    parameters.poly_degree = (short)hdr[3];
    parameters.cloud_size_multiplier = (short)hdr[4];
    parameters.num_vcycles = (short)hdr[6];
    parameters.num_relax = (short)hdr[7];
    parameters.num_levels = (short)nl;
    parameters.Re = flow[0];
    parameters.courant_number = flow[1];
    parameters.omega = (float)flow[2];
    parameters.poisson_solver_tolerance = 1e-10;
    parameters.rho = 1;
    parameters.mu = parameters.rho / parameters.Re;
    parameters.nu = parameters.mu / parameters.rho;
    mgm_reference_set_poisson_mode(hdr[8]);

    /* read_complete_mesh_data (mesh_functions.h:914-928), nodes from the file */
    PointStructure *ps = calloc(nl, sizeof(PointStructure));
    for (int l = 0; l < nl; l++) {
        int nn[2];
        rd(nn, sizeof(int), 2, f);
        PointStructure *p = &ps[l];
        p->poly_degree = parameters.poly_degree;
        calculate_parameters(p);
        AllocateMemoryPointStructure(p, nn[0]);
        rd(p->x, sizeof(double), nn[0], f);
        rd(p->y, sizeof(double), nn[0], f);
        rd(p->z, sizeof(double), nn[0], f);
        rd(p->x_normal, sizeof(double), nn[0], f);
        rd(p->y_normal, sizeof(double), nn[0], f);
        rd(p->z_normal, sizeof(double), nn[0], f);
        unsigned char *bt = malloc(nn[0]);
        rd(bt, 1, nn[0], f);
        for (int i = 0; i < nn[0]; i++) {
            p->boundary_tag[i] = bt[i] != 0;
            p->corner_tag[i] = false;
            p->point_index[i] = i;
        }
        free(bt);
        p->num_boundary_nodes = nn[1];
        p->num_corners = 0;
        find_cloud_index(p);
        rcm_reordering_with_boundarynodes(p);
        correct_normal_directions(p);
        calculate_avg_dx(p);
    }
    fclose(f);
    create_prolongation_and_restriction_matrices(ps, (short)nl);
    *out_ps = ps;
    return nl;
}

/* kind 0: fractional_step_explicit, 1: time_implicit_solver, 2: the step by routines */
static int run(PointStructure *ps, int nl, int nsteps, int kind, const char *out)
{
    const int timple = kind == 1;
    /* mg_NS_solver.c:47-59 with the lid-driven cavity conditions (init_LDC.c)
     * or, for TIMPLE, the Taylor-Couette ones (init_TC.c:33-52) */
    FieldVariables *field;
    AllocateMemoryFieldVariables(&field, ps, nl);
    for (int i = 0; i < ps[0].num_nodes; i++) {
        if (!timple) {
            if (fabs(ps[0].y[i] - 1.0) < 1e-9) field[0].u[i] = 1.0;
        } else {
            const double x = ps[0].x[i], y = ps[0].y[i], r = sqrt(x * x + y * y);
            if (fabs(r - 0.5) < 1e-9) {
                field[0].u[i] = -y / r; field[0].v[i] = x / r;
                field[0].u_new[i] = -y / r; field[0].v_new[i] = x / r;
            }
        }
    }
    if (timple) {
        parameters.iter_timple = 2;
        parameters.iter_momentum = 2;
        parameters.facRe = 1.0;
        parameters.facdt = 1.0;
    }
    parameters.dt = calculate_dt(&ps[0]);
    copyin_essentials_to_gpu(ps);
    copyin_field_to_gpu(field, ps);
    copyin_parameters_to_gpu();

    double *errs = malloc(sizeof(double) * (nsteps > 0 ? nsteps : 1));
    for (int s = 0; s < nsteps; s++) {
        if (kind == 2) {
            step_by_routines(ps, field, nl);
            errs[s] = 0;
        } else {
            errs[s] = timple ? time_implicit_solver(ps, field) : fractional_step_explicit(ps, field);
        }
    }

    for (int l = 0; l < nl; l++) {
        PointStructure *p = &ps[l];
        const int n = p->num_nodes, k = p->num_cloud_points;
        char nm[64];
        unsigned char *bt = malloc(n);
        for (int i = 0; i < n; i++) bt[i] = p->boundary_tag[i];
#define W(tag, ptr, bytes) do { snprintf(nm, sizeof(nm), "l%d_%s", l, tag); wr(out, nm, ptr, bytes); } while (0)
        W("x", p->x, sizeof(double) * n);
        W("y", p->y, sizeof(double) * n);
        W("nx", p->x_normal, sizeof(double) * n);
        W("ny", p->y_normal, sizeof(double) * n);
        W("btag", bt, n);
        W("d_avg", &p->d_avg, sizeof(double));
        W("rpts", p->restriction_points, sizeof(int) * n);
        W("ppts", p->prolongation_points, sizeof(int) * n);
#undef W
        snprintf(nm, sizeof(nm), "l%d_cloud", l); wr_rows_i(out, nm, p->cloud_index, n, k);
        snprintf(nm, sizeof(nm), "l%d_Dx", l); wr_rows_d(out, nm, p->Dx, n, k);
        snprintf(nm, sizeof(nm), "l%d_Dy", l); wr_rows_d(out, nm, p->Dy, n, k);
        snprintf(nm, sizeof(nm), "l%d_lap", l); wr_rows_d(out, nm, p->lap, n, k);
        snprintf(nm, sizeof(nm), "l%d_lapP", l); wr_rows_d(out, nm, p->lap_Poison, n, k);
        if (l > 0) { snprintf(nm, sizeof(nm), "l%d_restr", l); wr_rows_d(out, nm, p->restr_mat, n, ps[l - 1].num_cloud_points); }
        if (l < nl - 1) { snprintf(nm, sizeof(nm), "l%d_prol", l); wr_rows_d(out, nm, p->prol_mat, n, ps[l + 1].num_cloud_points); }
        free(bt);
    }
    wr(out, "dt", &parameters.dt, sizeof(double));
    wr(out, "errs", errs, sizeof(double) * nsteps);
    wr(out, "u", field[0].u, sizeof(double) * ps[0].num_nodes);
    wr(out, "v", field[0].v, sizeof(double) * ps[0].num_nodes);
    wr(out, "p", field[0].p, sizeof(double) * ps[0].num_nodes);
    wr(out, "u_new", field[0].u_new, sizeof(double) * ps[0].num_nodes);
    wr(out, "v_new", field[0].v_new, sizeof(double) * ps[0].num_nodes);
    wr(out, "p_old", field[0].p_old, sizeof(double) * ps[0].num_nodes);
    printf("legacy driver done: %d levels, %d steps\n", nl, nsteps);
    return 0;
}
