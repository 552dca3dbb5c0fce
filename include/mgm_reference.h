/*
 * mgm_reference.h -- drop-in replacement of the reference's C call surface
 * for the hot path (the Multigrid_meshless header_files), backed by the
 * sm_100a kernels of libmgm.so.
 *
 * A program written against the reference includes this header instead of
 * header_files/fractional_step_solver.h (+ openACC_functions.h) and links
 * -lmgm.  The structures below have the members, types and order of
 * header_files/structures.h:15-106 so that code filling or reading them is
 * unchanged; the global `parameters` is defined by the library.
 *
 * Differences from the reference, by design:
 *  - every function runs its compute on the GPU (no OpenACC, no CPU path);
 *  - node sets must be in the state read_PointStructure leaves them
 *    (boundary nodes first, no corner nodes); corner-tagged nodes are rejected;
 *  - exactly equal kNN distances are ordered by lower node index;
 *  - fatal errors print the library's message and exit(1), as the reference
 *    does on input errors (mesh_functions.h:43-47);
 *  - fractional_step_explicit keeps the fields on the device and copies the
 *    level-0 velocity, pressure and intermediate velocity back after each
 *    step (the reference's managed-memory view, mg_NS_solver.c:75).
 */
#ifndef MGM_REFERENCE_H
#define MGM_REFERENCE_H

/* The reference's structures.h guard: its init files (init/init_TC.c:7,
 * init/init_LDC.c:7) include "../header_files/structures.h", whose contents
 * this header replaces; with the guard defined that include adds nothing. */
#define STRUCTURES_H

#include <math.h>
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "mgm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* structures.h:15-41 */
struct parameters {
    short dimension;
    short poly_degree;
    short phs_degree;
    short cloud_size_multiplier;
    short test;
    double courant_number;
    double steady_state_tolerance;
    double poisson_solver_tolerance;
    short num_vcycles;
    short num_relax;
    int num_time_steps;
    short num_levels;
    int write_interval;
    bool neumann_flag_boundary;
    float omega;
    double dt;
    short iter_momentum;
    short iter_timple;
    double rho;
    double mu;
    double Re;
    double facRe;
    double facdt;
    double nu;
};
MGM_API extern struct parameters parameters;

/* structures.h:44-78 */
typedef struct PointStructure {
    char mesh_filename[50];
    int num_nodes;
    int num_corners;
    int num_boundary_nodes;
    int num_elem;
    double d_avg;
    short num_poly_terms;
    short num_cloud_points;
    short poly_degree;
    double *x;
    double *y;
    double *z;
    int *point_index;
    double *x_normal;
    double *y_normal;
    double *z_normal;
    bool *boundary_tag;
    bool *corner_tag;
    short *pow_x;
    short *pow_y;
    short *pow_z;
    int **cloud_index;
    int *prolongation_points;
    int *restriction_points;
    double **Dx;
    double **Dy;
    double **Dz;
    double **lap;
    double **lap_Poison;
    double **restr_mat;
    double **prol_mat;
    int **prolongation_points2;
    int **restriction_points2;
} PointStructure;

/* structures.h:80-106 */
typedef struct FieldVariables {
    double *u;
    double *v;
    double *w;
    double *p;
    double *u_new;
    double *v_new;
    double *w_new;
    double *u_old;
    double *v_old;
    double *w_old;
    double *p_old;
    double *pprime;
    double *res;
    double *source;
    double *T;
    double *dpdn;
    double *dpdx;
    double *dpdy;
    double *dpdz;
    double rho;
    double mu;
    double nu;
    double Re;
} FieldVariables;

/* structures.h:114-172 */
MGM_API void AllocateMemoryPointStructure(PointStructure *myPointStruct, int nodes);
MGM_API void AllocateMemoryFieldVariables(FieldVariables **field, PointStructure *myPointStruct, int num_levels);
/* structures.h:174-226: frees the levels' host arrays and jagged rows (rows
 * absent on a level are skipped, where the reference's version frees
 * unallocated restr_mat / prol_mat rows) and the device context when these
 * levels are the ones copyin_essentials_to_gpu took; free_field frees every
 * member array. */
MGM_API void free_PointStructure(PointStructure *myPointStruct, int num_levels);
MGM_API void free_field(FieldVariables *field, int num_levels);
/* general_functions.h:44-192: the derivative self-test (mg_NS_solver.c:40-43):
 * per level, the RMS error over interior nodes of Dx, Dy, (Dz), lap applied
 * on the GPU to sin(2*3.14*x) sin(2*3.14*y) (sin(2*3.14*z)) against its exact
 * derivatives, printed in the reference's format. */
MGM_API void test_derivatives(PointStructure *myPointStruct, short num_levels, short domain_dimension);
/* mesh_functions.h:37-129, 131-170 */
MGM_API void read_flow_parameters(char *filename);
MGM_API void read_grid_filenames(PointStructure **myPointStruct, char *filename, short *num_levels);
MGM_API void calculate_parameters(PointStructure *myPointStruct);
/* mesh_functions.h:172-476: the Gmsh reader (mgm_mesh_read) into the level's
 * arrays, corner nodes removed, num_boundary_nodes / num_elem / d_avg set. */
MGM_API void read_PointStructure(PointStructure *myPointStruct);
/* mesh_functions.h:914-928: per level read_PointStructure, find_cloud_index,
 * rcm_reordering_with_boundarynodes, correct_normal_directions,
 * calculate_avg_dx (poly_degree 3 on coarse levels, parameters.poly_degree on
 * the finest), then create_prolongation_and_restriction_matrices. */
MGM_API void read_complete_mesh_data(PointStructure *myPointStruct, short num_levels);
/* write_functions.h:29-201: text dumps of a level's host arrays, same formats
 * and file names (write_processed_grid_data writes the six per-level files
 * into the working directory). */
MGM_API void write_normals(PointStructure *myPointStruct, char *filename);
MGM_API void write_boundary_tags(PointStructure *myPointStruct, char *filename);
MGM_API void write_corner_tags(PointStructure *myPointStruct, char *filename);
MGM_API void write_coordinates(PointStructure *myPointStruct, char *filename);
MGM_API void write_cloud_index(PointStructure *myPointStruct, char *filename);
MGM_API void write_prolongation_and_restriction_points(PointStructure *myPointStruct, char *filename);
MGM_API void write_test_files(double *f, double *fx, double *fy, double *fz, double *lapf, double *fxx, double *fyy,
                              double *fzz, int num_nodes, char *folder1);
MGM_API void write_processed_grid_data(PointStructure *myPointStruct, int level);
/* kdtree_functions.h:113-175 */
MGM_API void find_cloud_index(PointStructure *myPointStruct1);
MGM_API int *find_nearest_point(PointStructure *myPointStruct1, PointStructure *myPointStruct2, int num_cloud_points);
/* mesh_functions.h:478-527, 533-670, 774-872, 874-910 */
MGM_API void rcm_reordering_with_boundarynodes(PointStructure *myPointstruct);
MGM_API void correct_normal_directions(PointStructure *myPointStruct);
MGM_API void calculate_avg_dx(PointStructure *myPointStruct);
MGM_API void create_restriction_matrix(PointStructure *myPointStruct_f, PointStructure *myPointStruct_c);
MGM_API void create_prolongation_matrix(PointStructure *myPointStruct_f, PointStructure *myPointStruct_c);
MGM_API void create_prolongation_and_restriction_matrices(PointStructure *myPointStruct, short num_levels);
/* rbf.h:32-40, 401-421 */
MGM_API double calculate_phs_rbf(double *pt1, double *pt2, int phs, int dimension);
MGM_API void create_derivative_matrices(PointStructure *myPointStruct);
/* rbf.h:274-380: one operator each (Dx, Dy, Dz, lap) into the level's rows
 * (allocated here when NULL); rbf.h:382-399: lap_Poison from lap, Dx, Dy,
 * (Dz) and the normals */
MGM_API void create_full_gradx_matrix(PointStructure *myPointStruct);
MGM_API void create_full_grady_matrix(PointStructure *myPointStruct);
MGM_API void create_full_gradz_matrix(PointStructure *myPointStruct);
MGM_API void create_full_laplacian_matrix(PointStructure *myPointStruct);
MGM_API void create_laplacian_for_Poisson(PointStructure *myPointStruct);
/* mat_lib.h:423-491 (order <= 1024), on the GPU; `inverse` rows allocated by the caller */
MGM_API void matrixInverse_Gauss_Jordan(double **matrix1, double **inverse, int order);
/* mat_lib.h:80-89 */
MGM_API void multiply_sparse_matrix_vector_gpu(double **D_coeff, double *f, double *dfdx, int **cloud, int n_rows_D,
                                               int n_cols_D);
/* general_functions.h:34-41 */
MGM_API double calculate_dt(PointStructure *myPointStruct);
/* openACC_functions.h:26-120 */
MGM_API void copyin_parameters_to_gpu(void);
MGM_API void copyin_essentials_to_gpu(PointStructure *myPointStruct);
MGM_API void copyin_field_to_gpu(FieldVariables *field, PointStructure *myPointStruct);
/* fractional_step_solver.h:28-37 */
MGM_API double fractional_step_explicit(PointStructure *myPointStruct, FieldVariables *field);
MGM_API void calculate_intermediate_velocity(PointStructure *myPointStruct, FieldVariables *field);
MGM_API void calculate_mass_residual(PointStructure *myPointStruct, FieldVariables *field);
MGM_API void calculate_boundary_dpdn(PointStructure *myPointStruct, FieldVariables *field);
MGM_API void multigrid_Poisson_solver(PointStructure *myPointStruct, FieldVariables *field);
/* fractional_step_solver.h:168-246: the multigrid's routines, on the device
 * levels of copyin_essentials_to_gpu (myPointStruct must point into that
 * array; restrict/prolongate take consecutive levels), sweeps in
 * data-parallel order; the device holds the fields, and the host arrays each
 * routine changes (p and res; the coarse source; both levels' p) are
 * refreshed after it runs. */
MGM_API void relaxation(PointStructure *myPointStruct, FieldVariables *field);
MGM_API void calculate_residuals(PointStructure *myPointStruct, FieldVariables *field);
MGM_API void restrict_residuals(PointStructure *myPointStruct_f, PointStructure *myPointStruct_c,
                                FieldVariables *field_f, FieldVariables *field_c);
MGM_API void prolongate_corrections(PointStructure *myPointStruct_f, PointStructure *myPointStruct_c,
                                    FieldVariables *field_f, FieldVariables *field_c);
MGM_API void update_velocity(PointStructure *myPointStruct, FieldVariables *field);

/* timple_solver.h:40-70, 72-201, 341-410 (the default solver of mg_NS_solver.c).
 * time_implicit_solver runs the TIMPLE variants of the multigrid routines
 * (timple_solver.h:203-339) internally; the exported multigrid_Poisson_solver,
 * relaxation, calculate_residuals, restrict_residuals and
 * prolongate_corrections above are the fractional step's.  Momentum sweeps run in
 * data-parallel order. */
MGM_API double time_implicit_solver(PointStructure *myPointStruct, FieldVariables *field);
MGM_API void calculate_intermediate_velocity_implicit(PointStructure *myPointStruct, FieldVariables *field);
MGM_API void calculate_mass_residual_implicit(PointStructure *myPointStruct, FieldVariables *field);
MGM_API void update_velocity_implicit(PointStructure *myPointStruct, FieldVariables *field);
MGM_API void update_boundary_pressure(PointStructure *myPointStruct, FieldVariables *field);

/* No counterpart in the reference: which Poisson solve multigrid_Poisson_solver
 * and fractional_step_explicit run (MGM_MODE_REFERENCE, the default: the
 * reference's fixed V-cycles; MGM_MODE_FP64 / MGM_MODE_FP32_IR: the
 * convergent solve to parameters.poisson_solver_tolerance). */
MGM_API void mgm_reference_set_poisson_mode(int mode);
/* No counterpart in the reference: mgm_set_compatible_rhs for the convergent
 * modes of mgm_reference_set_poisson_mode (the Poisson source projected along
 * lap_Poison's left null vector before the pinned solve); taken over by
 * copyin_essentials_to_gpu, and applied at once to a context already there. */
MGM_API void mgm_reference_set_compatible_rhs(int enable);

#ifdef __cplusplus
}
#endif
#endif
