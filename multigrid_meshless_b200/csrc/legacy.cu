// legacy.cu -- the reference's C call surface (include/mgm_reference.h) on top
// of the C ABI (include/mgm.h).  Host code only: it packs the reference's
// jagged rows into [n][k] arrays, calls the GPU entry points and unpacks the
// results into freshly malloc'd rows, as the reference's functions do.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mgm_reference.h"
#include "mgm_math.h"

struct parameters parameters;

namespace {

mgm_ctx *g_ctx = nullptr;
int g_levels = 0;
PointStructure *g_ps = nullptr;  // the level array handed to copyin_essentials_to_gpu
int g_mode = MGM_MODE_REFERENCE;
int g_compat = 0;  // mgm_reference_set_compatible_rhs

void die_if(int status, const char *what)
{
    if (status != MGM_OK) {
        std::printf("Error: %s: %s\n", what, mgm_last_error());
        std::exit(1);
    }
}

std::vector<unsigned char> tags(const bool *b, int n)
{
    std::vector<unsigned char> t(n);
    for (int i = 0; i < n; i++) t[i] = b[i] ? 1 : 0;
    return t;
}

std::vector<int> pack_rows(int *const *rows, int n, int k)
{
    std::vector<int> out((size_t)n * k);
    for (int i = 0; i < n; i++) std::memcpy(&out[(size_t)i * k], rows[i], sizeof(int) * k);
    return out;
}

std::vector<double> pack_rows(double *const *rows, int n, int k)
{
    std::vector<double> out((size_t)n * k);
    for (int i = 0; i < n; i++) std::memcpy(&out[(size_t)i * k], rows[i], sizeof(double) * k);
    return out;
}

template <class T>
T **unpack_rows(const std::vector<T> &flat, int n, int k)
{
    T **rows = (T **)std::malloc(sizeof(T *) * (size_t)n);
    for (int i = 0; i < n; i++) {
        rows[i] = (T *)std::malloc(sizeof(T) * (size_t)k);
        std::memcpy(rows[i], &flat[(size_t)i * k], sizeof(T) * k);
    }
    return rows;
}

void require_no_corners(const PointStructure *p, const char *fn)
{
    for (int i = 0; i < p->num_nodes; i++)
        if (p->corner_tag && p->corner_tag[i]) {
            std::printf("Error: %s: corner-tagged node %d present (remove corner nodes first, as read_PointStructure does)\n",
                        fn, i);
            std::exit(1);
        }
}

}  // namespace

extern "C" {

void mgm_reference_set_poisson_mode(int mode) { g_mode = mode; }

void mgm_reference_set_compatible_rhs(int enable)
{
    g_compat = enable != 0;
    if (g_ctx) die_if(mgm_set_compatible_rhs(g_ctx, g_compat), "mgm_reference_set_compatible_rhs");
}

// structures.h:114-126
void AllocateMemoryPointStructure(PointStructure *p, int nodes)
{
    p->x_normal = (double *)std::malloc(nodes * sizeof(double));
    p->y_normal = (double *)std::malloc(nodes * sizeof(double));
    p->z_normal = (double *)std::malloc(nodes * sizeof(double));
    p->x = (double *)std::malloc(nodes * sizeof(double));
    p->y = (double *)std::malloc(nodes * sizeof(double));
    p->z = (double *)std::malloc(nodes * sizeof(double));
    p->point_index = (int *)std::malloc(nodes * sizeof(int));
    p->boundary_tag = (bool *)std::malloc(nodes * sizeof(bool));
    p->corner_tag = (bool *)std::malloc(nodes * sizeof(bool));
    p->num_nodes = nodes;
    p->num_elem = 0;
}

// structures.h:128-172: every member array zero-filled
void AllocateMemoryFieldVariables(FieldVariables **field, PointStructure *ps, int num_levels)
{
    *field = (FieldVariables *)std::calloc((size_t)num_levels, sizeof(FieldVariables));
    for (int l = 0; l < num_levels; l++) {
        const size_t n = (size_t)ps[l].num_nodes;
        FieldVariables *f = &(*field)[l];
        double **arrs[] = {&f->u, &f->v, &f->w, &f->u_new, &f->v_new, &f->w_new, &f->pprime, &f->p, &f->u_old,
                           &f->v_old, &f->w_old, &f->p_old, &f->res, &f->source, &f->dpdn, &f->dpdx, &f->dpdy,
                           &f->dpdz, &f->T};
        for (double **a : arrs) *a = (double *)std::calloc(n, sizeof(double));
    }
}

// mesh_functions.h:37-100: positional "name,value" lines in this order
void read_flow_parameters(char *filename)
{
    FILE *f = std::fopen(filename, "r");
    if (!f) { std::printf("Error: Unable to open the file\n"); std::exit(1); }
    char name[100];
    int itmp = 0, r = 0;
    r = std::fscanf(f, "%[^,],%hd\n", name, &parameters.dimension);
    r = std::fscanf(f, "%[^,],%hd\n", name, &parameters.poly_degree);
    r = std::fscanf(f, "%[^,],%hd\n", name, &parameters.phs_degree);
    r = std::fscanf(f, "%[^,],%hd\n", name, &parameters.cloud_size_multiplier);
    r = std::fscanf(f, "%[^,],%hd\n", name, &parameters.test);
    r = std::fscanf(f, "%[^,],%lf\n", name, &parameters.courant_number);
    r = std::fscanf(f, "%[^,],%lf\n", name, &parameters.steady_state_tolerance);
    r = std::fscanf(f, "%[^,],%lf\n", name, &parameters.poisson_solver_tolerance);
    r = std::fscanf(f, "%[^,],%f\n", name, &parameters.omega);
    r = std::fscanf(f, "%[^,],%hd\n", name, &parameters.num_vcycles);
    r = std::fscanf(f, "%[^,],%hd\n", name, &parameters.num_relax);
    r = std::fscanf(f, "%[^,],%d\n", name, &parameters.num_time_steps);
    r = std::fscanf(f, "%[^,],%d\n", name, &parameters.write_interval);
    r = std::fscanf(f, "%[^,],%d\n", name, &itmp);
    parameters.neumann_flag_boundary = itmp == 1;
    r = std::fscanf(f, "%[^,],%lf\n", name, &parameters.dt);
    r = std::fscanf(f, "%[^,],%hd\n", name, &parameters.iter_momentum);
    r = std::fscanf(f, "%[^,],%hd\n", name, &parameters.iter_timple);
    r = std::fscanf(f, "%[^,],%lf\n", name, &parameters.Re);
    r = std::fscanf(f, "%[^,],%lf\n", name, &parameters.facRe);
    r = std::fscanf(f, "%[^,],%lf\n", name, &parameters.facdt);
    std::fclose(f);
    if (r == EOF) { std::printf("Error: Unable to read the file\n"); std::exit(1); }
    parameters.rho = 1;
    parameters.mu = parameters.rho / parameters.Re;
    parameters.nu = parameters.mu / parameters.rho;
}

// mesh_functions.h:102-129
void read_grid_filenames(PointStructure **ps, char *filename, short *num_levels)
{
    FILE *f = std::fopen(filename, "r");
    if (!f) { std::printf("Error: Unable to open the file\n"); std::exit(1); }
    char name[100];
    if (std::fscanf(f, "%[^,],%hd\n", name, num_levels) == EOF) { std::printf("Error: Unable to read the file\n"); std::exit(1); }
    *ps = (PointStructure *)std::calloc((size_t)*num_levels, sizeof(PointStructure));
    for (short l = 0; l < *num_levels; l++)
        if (std::fscanf(f, "%49s\n", (*ps)[l].mesh_filename) == EOF) {
            std::printf("Error: Unable to read the meshfile names\n");
            std::exit(1);
        }
    std::fclose(f);
}

// ---- write_functions.h:29-201: text dumps of a level (same formats) ----
static std::FILE *open_or_exit(const char *filename)
{
    std::FILE *f = std::fopen(filename, "w");
    if (!f) {
        std::printf("Error: Unable to open the file %s\n", filename);
        std::exit(1);
    }
    return f;
}

void write_normals(PointStructure *p, char *filename)
{
    std::printf("Writing normals to file %s\n", filename);
    std::FILE *f = open_or_exit(filename);
    for (int i = 0; i < p->num_nodes; i++)
        std::fprintf(f, "%d %lf %lf %lf\n", i, p->x_normal[i], p->y_normal[i], p->z_normal[i]);
    std::fclose(f);
}

void write_boundary_tags(PointStructure *p, char *filename)
{
    std::printf("Writing boundary tags to file %s\n", filename);
    std::FILE *f = open_or_exit(filename);
    for (int i = 0; i < p->num_nodes; i++) std::fprintf(f, "%d %d\n", i, (int)p->boundary_tag[i]);
    std::fclose(f);
}

void write_corner_tags(PointStructure *p, char *filename)
{
    std::printf("Writing corner tags to file %s\n", filename);
    std::FILE *f = open_or_exit(filename);
    for (int i = 0; i < p->num_nodes; i++) std::fprintf(f, "%d %d\n", i, (int)p->corner_tag[i]);
    std::fclose(f);
}

void write_coordinates(PointStructure *p, char *filename)
{
    std::printf("Writing coordinates to %s\n", filename);
    std::FILE *f = open_or_exit(filename);
    for (int i = 0; i < p->num_nodes; i++) std::fprintf(f, "%lf %lf %lf\n", p->x[i], p->y[i], p->z[i]);
    std::fclose(f);
}

void write_cloud_index(PointStructure *p, char *filename)
{
    std::printf("Writing cloud index to %s\n", filename);
    std::FILE *f = open_or_exit(filename);
    for (int i = 0; i < p->num_nodes; i++) {
        std::fprintf(f, "%d ", i);
        for (int j = 0; j < p->num_cloud_points; j++) std::fprintf(f, "%d ", p->cloud_index[i][j]);
        std::fprintf(f, "\n");
    }
    std::fclose(f);
}

void write_prolongation_and_restriction_points(PointStructure *p, char *filename)
{
    std::printf("Writing prolongation and restriction points to %s\n", filename);
    std::FILE *f = open_or_exit(filename);
    for (int i = 0; i < p->num_nodes; i++)
        std::fprintf(f, "%d %d %d\n", i, p->prolongation_points[i], p->restriction_points[i]);
    std::fclose(f);
}

// folder1 is a prefix (the reference concatenates it with the file names in a
// 100-character buffer)
void write_test_files(double *f, double *fx, double *fy, double *fz, double *lapf, double *fxx, double *fyy,
                      double *fzz, int num_nodes, char *folder1)
{
    const char *names[8] = {"f.csv", "fx.csv", "fy.csv", "fz.csv", "lapf.csv", "fxx.csv", "fyy.csv", "fzz.csv"};
    double *arrs[8] = {f, fx, fy, fz, lapf, fxx, fyy, fzz};
    for (int t = 0; t < 8; t++) {
        std::string path = std::string(folder1) + names[t];
        std::FILE *o = std::fopen(path.c_str(), "w");
        if (!o) {
            std::printf("Error: Unable to open the file %s\n", path.c_str());
            std::exit(1);
        }
        for (int i = 0; i < num_nodes; i++) std::fprintf(o, "%f\n", arrs[t][i]);
        std::fclose(o);
    }
    std::printf("Files written\n");
}

void write_processed_grid_data(PointStructure *p, int level)
{
    char name[64];
    std::snprintf(name, sizeof(name), "normals_%d.csv", level);
    write_normals(p, name);
    std::snprintf(name, sizeof(name), "boundary_tags_%d.csv", level);
    write_boundary_tags(p, name);
    std::snprintf(name, sizeof(name), "corner_tags_%d.csv", level);
    write_corner_tags(p, name);
    std::snprintf(name, sizeof(name), "coordinates_%d.csv", level);
    write_coordinates(p, name);
    std::snprintf(name, sizeof(name), "cloud_index_%d.csv", level);
    write_cloud_index(p, name);
    std::snprintf(name, sizeof(name), "prolongation_and_restriction_%d.csv", level);
    write_prolongation_and_restriction_points(p, name);
    std::printf("\n\n");
}

// mesh_functions.h:172-476, through mgm_mesh_read (the same messages on stdout)
void read_PointStructure(PointStructure *p)
{
    mgm_mesh *m = nullptr;
    die_if(mgm_mesh_read(p->mesh_filename, parameters.dimension, &m), "read_PointStructure");
    int n = 0, nb = 0, ne = 0;
    double d_avg = 0;
    die_if(mgm_mesh_info(m, &n, &nb, &ne, &d_avg), "read_PointStructure");
    AllocateMemoryPointStructure(p, n);
    std::vector<unsigned char> bt(n), ct(n);
    die_if(mgm_mesh_get(m, p->x, p->y, p->z, p->x_normal, p->y_normal, p->z_normal, bt.data(), ct.data()),
           "read_PointStructure");
    mgm_mesh_free(m);
    for (int i = 0; i < n; i++) {
        p->boundary_tag[i] = bt[i] != 0;
        p->corner_tag[i] = ct[i] != 0;
        p->point_index[i] = i;
    }
    p->num_elem = ne;
    p->d_avg = d_avg;
    p->num_boundary_nodes = nb;
    p->num_corners = 0;
    std::printf("Average distance between nodes = %lf\n", d_avg);
    std::printf("No of nodes = %d \nNo of elements = %d \n", n, ne);
    std::printf("No of boundary nodes = %d \nNo of corner nodes = %d \n", nb, 0);
}

// mesh_functions.h:914-928
void read_complete_mesh_data(PointStructure *ps, short num_levels)
{
    for (short l = 0; l < num_levels; l++) {
        ps[l].poly_degree = 3;
        ps[0].poly_degree = parameters.poly_degree;
        std::printf("\nReading mesh data for level %d\n", l + 1);
        calculate_parameters(&ps[l]);
        read_PointStructure(&ps[l]);
        find_cloud_index(&ps[l]);
        rcm_reordering_with_boundarynodes(&ps[l]);
        correct_normal_directions(&ps[l]);
        calculate_avg_dx(&ps[l]);
    }
    create_prolongation_and_restriction_matrices(ps, num_levels);
}

// mesh_functions.h:131-170
void calculate_parameters(PointStructure *p)
{
    const int d = p->poly_degree;
    p->num_poly_terms = parameters.dimension == 3 ? (d + 1) * (d + 2) * (d + 3) / 6 : (d + 1) * (d + 2) / 2;
    p->num_cloud_points = parameters.cloud_size_multiplier * p->num_poly_terms;
    p->pow_x = (short *)std::malloc(p->num_poly_terms * sizeof(short));
    p->pow_y = (short *)std::malloc(p->num_poly_terms * sizeof(short));
    p->pow_z = (short *)std::malloc(p->num_poly_terms * sizeof(short));
    int c = 0;
    for (int i = 0; i <= d; i++)
        for (int j = 0; j <= d - i; j++) {
            if (parameters.dimension == 3) {
                for (int l = 0; l <= d - i - j; l++) { p->pow_x[c] = i; p->pow_y[c] = j; p->pow_z[c] = l; c++; }
            } else { p->pow_x[c] = i; p->pow_y[c] = j; p->pow_z[c] = 0; c++; }
        }
}

void find_cloud_index(PointStructure *p)
{
    require_no_corners(p, "find_cloud_index");
    const int n = p->num_nodes, k = p->num_cloud_points;
    std::vector<unsigned char> bt = tags(p->boundary_tag, n);
    std::vector<int> cl((size_t)n * k);
    die_if(mgm_knn_cloud(n, p->num_boundary_nodes, parameters.dimension, p->x, p->y, p->z, bt.data(), k, cl.data()),
           "find_cloud_index");
    p->cloud_index = unpack_rows(cl, n, k);
}

int *find_nearest_point(PointStructure *p1, PointStructure *p2, int num_cloud_points)
{
    (void)num_cloud_points;  // the reference asks for 3 and keeps the first
    int *out = (int *)std::malloc(sizeof(int) * (size_t)p1->num_nodes);
    die_if(mgm_nearest_points(p1->num_nodes, p1->x, p1->y, p1->z, p2->num_nodes, p2->x, p2->y, p2->z,
                              parameters.dimension, out),
           "find_nearest_point");
    return out;
}

void rcm_reordering_with_boundarynodes(PointStructure *p)
{
    const int n = p->num_nodes, k = p->num_cloud_points;
    std::vector<int> cl = pack_rows(p->cloud_index, n, k), q1(n);
    die_if(mgm_bfs_order(n, k, cl.data(), q1.data()), "rcm_reordering_with_boundarynodes");
    std::vector<unsigned char> bt = tags(p->boundary_tag, n);
    die_if(mgm_apply_order(n, k, q1.data(), p->x, p->y, p->z, p->x_normal, p->y_normal, p->z_normal, bt.data(),
                           cl.data()),
           "rcm_reordering_with_boundarynodes");
    for (int i = 0; i < n; i++) {
        p->boundary_tag[i] = bt[i] != 0;
        std::memcpy(p->cloud_index[i], &cl[(size_t)i * k], sizeof(int) * k);
    }
}

void correct_normal_directions(PointStructure *p)
{
    const int n = p->num_nodes, k = p->num_cloud_points;
    std::vector<int> cl = pack_rows(p->cloud_index, n, k);
    std::vector<unsigned char> bt = tags(p->boundary_tag, n);
    die_if(mgm_correct_normals(n, k, p->x, p->y, p->z, bt.data(), cl.data(), p->x_normal, p->y_normal, p->z_normal),
           "correct_normal_directions");
}

void calculate_avg_dx(PointStructure *p)
{
    const int n = p->num_nodes, k = p->num_cloud_points;
    std::vector<int> cl = pack_rows(p->cloud_index, n, k);
    std::vector<unsigned char> bt = tags(p->boundary_tag, n);
    die_if(mgm_avg_dx(n, k, parameters.dimension, p->x, p->y, p->z, bt.data(), cl.data(), &p->d_avg), "calculate_avg_dx");
}

void create_restriction_matrix(PointStructure *f, PointStructure *c)
{
    const int kf = f->num_cloud_points;
    std::vector<int> scl = pack_rows(f->cloud_index, f->num_nodes, kf);
    std::vector<unsigned char> bt = tags(c->boundary_tag, c->num_nodes);
    std::vector<double> W((size_t)c->num_nodes * kf);
    die_if(mgm_transfer_weights(c->num_nodes, c->x, c->y, c->z, bt.data(), c->restriction_points, c->num_boundary_nodes,
                                0, f->num_nodes, kf, parameters.dimension, parameters.phs_degree, f->poly_degree, f->x,
                                f->y, f->z, scl.data(), W.data()),
           "create_restriction_matrix");
    c->restr_mat = unpack_rows(W, c->num_nodes, kf);
}

void create_prolongation_matrix(PointStructure *f, PointStructure *c)
{
    const int kc = c->num_cloud_points;
    std::vector<int> scl = pack_rows(c->cloud_index, c->num_nodes, kc);
    std::vector<unsigned char> bt = tags(f->boundary_tag, f->num_nodes);
    std::vector<double> W((size_t)f->num_nodes * kc);
    die_if(mgm_transfer_weights(f->num_nodes, f->x, f->y, f->z, bt.data(), f->prolongation_points, f->num_boundary_nodes,
                                0, c->num_nodes, kc, parameters.dimension, parameters.phs_degree, c->poly_degree, c->x,
                                c->y, c->z, scl.data(), W.data()),
           "create_prolongation_matrix");
    f->prol_mat = unpack_rows(W, f->num_nodes, kc);
}

// mesh_functions.h:874-893
void create_prolongation_and_restriction_matrices(PointStructure *ps, short num_levels)
{
    for (short l = 0; l < num_levels; l++) {
        if (l == num_levels - 1) ps[l].prolongation_points = find_nearest_point(&ps[l], &ps[l], 1);
        else {
            ps[l].prolongation_points = find_nearest_point(&ps[l], &ps[l + 1], 1);
            create_prolongation_matrix(&ps[l], &ps[l + 1]);
        }
        if (l == 0) ps[l].restriction_points = find_nearest_point(&ps[l], &ps[l], 1);
        else {
            ps[l].restriction_points = find_nearest_point(&ps[l], &ps[l - 1], 1);
            create_restriction_matrix(&ps[l - 1], &ps[l]);
        }
    }
}

double calculate_phs_rbf(double *pt1, double *pt2, int phs, int dimension)
{
    return mgm_phs_rbf(pt1, pt2, phs, dimension);
}

void create_derivative_matrices(PointStructure *p)
{
    require_no_corners(p, "create_derivative_matrices");
    const int n = p->num_nodes, k = p->num_cloud_points, dim = parameters.dimension;
    std::vector<int> cl = pack_rows(p->cloud_index, n, k);
    std::vector<unsigned char> bt = tags(p->boundary_tag, n);
    std::vector<double> Dx((size_t)n * k), Dy((size_t)n * k), Dz(dim == 3 ? (size_t)n * k : 0), lap((size_t)n * k),
        lapP((size_t)n * k);
    die_if(mgm_derivative_weights(n, k, dim, parameters.phs_degree, p->poly_degree, p->x, p->y, p->z, p->x_normal,
                                  p->y_normal, p->z_normal, bt.data(), cl.data(), Dx.data(), Dy.data(),
                                  dim == 3 ? Dz.data() : nullptr, lap.data(), lapP.data()),
           "create_derivative_matrices");
    p->Dx = unpack_rows(Dx, n, k);
    p->Dy = unpack_rows(Dy, n, k);
    p->Dz = dim == 3 ? unpack_rows(Dz, n, k) : nullptr;
    p->lap = unpack_rows(lap, n, k);
    p->lap_Poison = unpack_rows(lapP, n, k);
}

// create_full_gradx/grady/gradz/laplacian_matrix (rbf.h:274-380): one operator
// of the level into its (caller-allocated, or here allocated) rows
static void full_operator(PointStructure *p, int which, const char *fn)
{
    require_no_corners(p, fn);
    const int n = p->num_nodes, k = p->num_cloud_points, dim = parameters.dimension;
    if (which == 2 && dim != 3) return;
    std::vector<int> cl = pack_rows(p->cloud_index, n, k);
    std::vector<unsigned char> bt = tags(p->boundary_tag, n);
    std::vector<double> op[5];
    for (int t = 0; t < 5; t++) op[t].resize(t == 2 && dim != 3 ? 0 : (size_t)n * k);
    die_if(mgm_derivative_weights(n, k, dim, parameters.phs_degree, p->poly_degree, p->x, p->y, p->z, p->x_normal,
                                  p->y_normal, p->z_normal, bt.data(), cl.data(), op[0].data(), op[1].data(),
                                  dim == 3 ? op[2].data() : nullptr, op[3].data(), op[4].data()),
           fn);
    double ***dst[4] = {&p->Dx, &p->Dy, &p->Dz, &p->lap};
    if (!*dst[which]) *dst[which] = unpack_rows(op[which], n, k);
    else
        for (int i = 0; i < n; i++) std::memcpy((*dst[which])[i], &op[which][(size_t)i * k], sizeof(double) * k);
}
void create_full_gradx_matrix(PointStructure *p) { full_operator(p, 0, "create_full_gradx_matrix"); }
void create_full_grady_matrix(PointStructure *p) { full_operator(p, 1, "create_full_grady_matrix"); }
void create_full_gradz_matrix(PointStructure *p) { full_operator(p, 2, "create_full_gradz_matrix"); }
void create_full_laplacian_matrix(PointStructure *p) { full_operator(p, 3, "create_full_laplacian_matrix"); }

// rbf.h:382-399, from the level's Dx, Dy, (Dz), lap and normals
void create_laplacian_for_Poisson(PointStructure *p)
{
    const int n = p->num_nodes, k = p->num_cloud_points, dim = parameters.dimension;
    std::vector<unsigned char> bt = tags(p->boundary_tag, n);
    std::vector<double> Dx = pack_rows(p->Dx, n, k), Dy = pack_rows(p->Dy, n, k), lap = pack_rows(p->lap, n, k),
                        Dz, out((size_t)n * k);
    if (dim == 3) Dz = pack_rows(p->Dz, n, k);
    die_if(mgm_laplacian_for_poisson(n, k, dim, Dx.data(), Dy.data(), dim == 3 ? Dz.data() : nullptr, lap.data(),
                                     p->x_normal, p->y_normal, p->z_normal, bt.data(), out.data()),
           "create_laplacian_for_Poisson");
    if (!p->lap_Poison) p->lap_Poison = unpack_rows(out, n, k);
    else
        for (int i = 0; i < n; i++) std::memcpy(p->lap_Poison[i], &out[(size_t)i * k], sizeof(double) * k);
}

// mat_lib.h:423-491 on the GPU; inverse rows allocated by the caller
void matrixInverse_Gauss_Jordan(double **matrix1, double **inverse, int order)
{
    std::vector<double> a = pack_rows(matrix1, order, order), inv((size_t)order * order);
    die_if(mgm_gauss_jordan(order, a.data(), inv.data()), "matrixInverse_Gauss_Jordan");
    for (int i = 0; i < order; i++) std::memcpy(inverse[i], &inv[(size_t)i * order], sizeof(double) * order);
}

void multiply_sparse_matrix_vector_gpu(double **D, double *f, double *dfdx, int **cloud, int n, int k)
{
    std::vector<double> W = pack_rows(D, n, k);
    std::vector<int> cl = pack_rows(cloud, n, k);
    die_if(mgm_spmv(n, k, W.data(), cl.data(), f, dfdx), "multiply_sparse_matrix_vector_gpu");
}

// general_functions.h:34-41
double calculate_dt(PointStructure *p)
{
    const double d = p->d_avg;
    const double termd = 2 * parameters.nu / (d * d);
    const double termc = 1 / d;
    const double dt = 0.5 / (termd + termc);
    return dt * parameters.courant_number;
}

void copyin_parameters_to_gpu(void)
{
    if (g_ctx)
        die_if(mgm_set_flow(g_ctx, parameters.Re, parameters.courant_number, parameters.omega, parameters.num_relax,
                            parameters.num_vcycles, parameters.dt),
               "copyin_parameters_to_gpu");
}

// openACC_functions.h:96-120: the level data of every level on the device
void copyin_essentials_to_gpu(PointStructure *ps)
{
    if (g_ctx) mgm_destroy(g_ctx);
    g_levels = parameters.num_levels;
    g_ps = ps;
    g_ctx = mgm_create(parameters.dimension, parameters.phs_degree, g_levels);
    if (!g_ctx) { std::printf("Error: copyin_essentials_to_gpu: %s\n", mgm_last_error()); std::exit(1); }
    for (int l = 0; l < g_levels; l++) {
        PointStructure *p = &ps[l];
        const int n = p->num_nodes, k = p->num_cloud_points;
        std::vector<int> cl = pack_rows(p->cloud_index, n, k);
        std::vector<unsigned char> bt = tags(p->boundary_tag, n);
        std::vector<double> Dx = pack_rows(p->Dx, n, k), Dy = pack_rows(p->Dy, n, k), lap = pack_rows(p->lap, n, k),
                            lapP = pack_rows(p->lap_Poison, n, k);
        std::vector<double> Dz;
        if (parameters.dimension == 3) Dz = pack_rows(p->Dz, n, k);
        die_if(mgm_load_level(g_ctx, l, n, p->num_boundary_nodes, p->x, p->y, p->z, p->x_normal, p->y_normal,
                              p->z_normal, bt.data(), p->poly_degree, k, cl.data(), Dx.data(), Dy.data(),
                              parameters.dimension == 3 ? Dz.data() : nullptr, lap.data(), lapP.data(),
                              p->restriction_points, p->prolongation_points, p->d_avg),
               "copyin_essentials_to_gpu");
    }
    for (int l = 0; l < g_levels; l++) {
        PointStructure *p = &ps[l];
        std::vector<double> restr, prol;
        if (l > 0 && p->restr_mat) restr = pack_rows(p->restr_mat, p->num_nodes, ps[l - 1].num_cloud_points);
        if (l < g_levels - 1 && p->prol_mat) prol = pack_rows(p->prol_mat, p->num_nodes, ps[l + 1].num_cloud_points);
        die_if(mgm_load_transfer(g_ctx, l, restr.empty() ? nullptr : restr.data(), prol.empty() ? nullptr : prol.data()),
               "copyin_essentials_to_gpu");
    }
    die_if(mgm_prepare(g_ctx), "copyin_essentials_to_gpu");
    die_if(mgm_set_solver(g_ctx, parameters.poisson_solver_tolerance > 0 ? parameters.poisson_solver_tolerance : 1e-8,
                          100, 4, 10.0),
           "copyin_essentials_to_gpu");
    if (g_compat) die_if(mgm_set_compatible_rhs(g_ctx, 1), "copyin_essentials_to_gpu");
}

// openACC_functions.h:67-90: level-0 fields (the coarse levels start at zero, as allocated)
void copyin_field_to_gpu(FieldVariables *field, PointStructure *ps)
{
    (void)ps;
    if (!g_ctx) { std::printf("Error: copyin_field_to_gpu before copyin_essentials_to_gpu\n"); std::exit(1); }
    copyin_parameters_to_gpu();
    const FieldVariables *f = &field[0];
    die_if(mgm_set_field(g_ctx, 0, MGM_FIELD_U, f->u), "copyin_field_to_gpu");
    die_if(mgm_set_field(g_ctx, 0, MGM_FIELD_V, f->v), "copyin_field_to_gpu");
    die_if(mgm_set_field(g_ctx, 0, MGM_FIELD_W, f->w), "copyin_field_to_gpu");
    die_if(mgm_set_field(g_ctx, 0, MGM_FIELD_U_NEW, f->u_new), "copyin_field_to_gpu");
    die_if(mgm_set_field(g_ctx, 0, MGM_FIELD_V_NEW, f->v_new), "copyin_field_to_gpu");
    die_if(mgm_set_field(g_ctx, 0, MGM_FIELD_P, f->p), "copyin_field_to_gpu");
    die_if(mgm_set_field(g_ctx, 0, MGM_FIELD_SOURCE, f->source), "copyin_field_to_gpu");
    // the TIMPLE step's state (timple_solver.h): w_new and the pressure p_old
    die_if(mgm_set_field(g_ctx, 0, MGM_FIELD_W_NEW, f->w_new), "copyin_field_to_gpu");
    die_if(mgm_set_field(g_ctx, 0, MGM_FIELD_P_OLD, f->p_old), "copyin_field_to_gpu");
}

static void need_ctx(const char *fn)
{
    if (!g_ctx) { std::printf("Error: %s before copyin_essentials_to_gpu\n", fn); std::exit(1); }
}

// the level index of a PointStructure of the array handed to copyin_essentials_to_gpu
static int level_of(const PointStructure *p, const char *fn)
{
    need_ctx(fn);
    const long l = p - g_ps;
    if (!g_ps || l < 0 || l >= g_levels) {
        std::printf("Error: %s: not a level of the structure passed to copyin_essentials_to_gpu\n", fn);
        std::exit(1);
    }
    return (int)l;
}

// fractional_step_solver.h:168-246: one multigrid routine on the device levels
// (data-parallel sweep order); the host arrays it changes are refreshed after
void relaxation(PointStructure *p, FieldVariables *f)
{
    const int l = level_of(p, "relaxation");
    die_if(mgm_ref_routine(g_ctx, l, MGM_REF_RELAXATION), "relaxation");
    die_if(mgm_get_field(g_ctx, l, MGM_FIELD_P, f->p), "relaxation");
    die_if(mgm_get_field(g_ctx, l, MGM_FIELD_RES, f->res), "relaxation");
}

void calculate_residuals(PointStructure *p, FieldVariables *f)
{
    const int l = level_of(p, "calculate_residuals");
    die_if(mgm_ref_routine(g_ctx, l, MGM_REF_RESIDUALS), "calculate_residuals");
    die_if(mgm_get_field(g_ctx, l, MGM_FIELD_RES, f->res), "calculate_residuals");
}

void restrict_residuals(PointStructure *pf, PointStructure *pc, FieldVariables *ff, FieldVariables *fc)
{
    (void)ff;
    const int l = level_of(pf, "restrict_residuals");
    if (pc != pf + 1) { std::printf("Error: restrict_residuals: levels not consecutive\n"); std::exit(1); }
    die_if(mgm_ref_routine(g_ctx, l, MGM_REF_RESTRICT), "restrict_residuals");
    die_if(mgm_get_field(g_ctx, l + 1, MGM_FIELD_SOURCE, fc->source), "restrict_residuals");
}

void prolongate_corrections(PointStructure *pf, PointStructure *pc, FieldVariables *ff, FieldVariables *fc)
{
    const int l = level_of(pf, "prolongate_corrections");
    if (pc != pf + 1) { std::printf("Error: prolongate_corrections: levels not consecutive\n"); std::exit(1); }
    die_if(mgm_ref_routine(g_ctx, l, MGM_REF_PROLONGATE), "prolongate_corrections");
    die_if(mgm_get_field(g_ctx, l, MGM_FIELD_P, ff->p), "prolongate_corrections");
    die_if(mgm_get_field(g_ctx, l + 1, MGM_FIELD_P, fc->p), "prolongate_corrections");
}

void calculate_intermediate_velocity(PointStructure *p, FieldVariables *f)
{
    (void)p;
    need_ctx("calculate_intermediate_velocity");
    die_if(mgm_intermediate_velocity(g_ctx), "calculate_intermediate_velocity");
    // `acc update host(u_new, v_new)` (fractional_step_solver.h:113)
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_U_NEW, f->u_new), "calculate_intermediate_velocity");
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_V_NEW, f->v_new), "calculate_intermediate_velocity");
}

void calculate_mass_residual(PointStructure *p, FieldVariables *f)
{
    (void)p; (void)f;
    need_ctx("calculate_mass_residual");
    die_if(mgm_mass_residual(g_ctx), "calculate_mass_residual");  // also writes the boundary dp/dn
}

void calculate_boundary_dpdn(PointStructure *p, FieldVariables *f)
{
    (void)p; (void)f;  // computed together with the mass residual (one pass over the stencils)
}

void multigrid_Poisson_solver(PointStructure *p, FieldVariables *f)
{
    (void)p; (void)f;
    need_ctx("multigrid_Poisson_solver");
    die_if(mgm_poisson(g_ctx, g_mode), "multigrid_Poisson_solver");
}

void update_velocity(PointStructure *p, FieldVariables *f)
{
    need_ctx("update_velocity");
    double mass = 0;
    die_if(mgm_update_velocity(g_ctx, &mass), "update_velocity");
    std::printf("Mass residual: %e\n", mass);
    // the host view of the corrected velocities (the reference's managed memory)
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_U, f->u), "update_velocity");
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_V, f->v), "update_velocity");
    if (parameters.dimension == 3) die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_W, f->w), "update_velocity");
    (void)p;
}

// fractional_step_solver.h:47-71
double fractional_step_explicit(PointStructure *ps, FieldVariables *field)
{
    need_ctx("fractional_step_explicit");
    FieldVariables *f = &field[0];
    const int n = ps[0].num_nodes;
    std::memcpy(f->u_old, f->u, sizeof(double) * n);
    std::memcpy(f->v_old, f->v, sizeof(double) * n);
    if (parameters.dimension == 3) std::memcpy(f->w_old, f->w, sizeof(double) * n);
    calculate_intermediate_velocity(&ps[0], f);
    calculate_mass_residual(&ps[0], f);
    calculate_boundary_dpdn(&ps[0], f);
    multigrid_Poisson_solver(ps, field);
    update_velocity(&ps[0], f);
    double err = 0;
    die_if(mgm_last_steady_error(g_ctx, &err), "fractional_step_explicit");
    // managed-memory view of level 0 (mg_NS_solver.c:75)
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_U, f->u), "fractional_step_explicit");
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_V, f->v), "fractional_step_explicit");
    if (parameters.dimension == 3) die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_W, f->w), "fractional_step_explicit");
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_P, f->p), "fractional_step_explicit");
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_SOURCE, f->source), "fractional_step_explicit");
    return err;
}

// ---------------------------------------------------------------------------
// the time-implicit solver (header_files/timple_solver.h), the default of
// mg_NS_solver.c.  Its multigrid_Poisson_solver / relaxation / ... share their
// names with the fractional step's; this library's exports of those names
// are the fractional step's, and time_implicit_solver runs the TIMPLE
// variants internally.
// ---------------------------------------------------------------------------
static void timple_params()
{
    die_if(mgm_set_timple(g_ctx, parameters.iter_timple > 0 ? parameters.iter_timple : 1,
                          parameters.iter_momentum > 0 ? parameters.iter_momentum : 1, parameters.facRe,
                          parameters.facdt > 0 ? parameters.facdt : 1.0),
           "TIMPLE parameters");
}

static void timple_host_view(FieldVariables *f, int n)
{
    (void)n;
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_U_NEW, f->u_new), "TIMPLE fields");
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_V_NEW, f->v_new), "TIMPLE fields");
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_U, f->u), "TIMPLE fields");
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_V, f->v), "TIMPLE fields");
    if (parameters.dimension == 3) {
        die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_W_NEW, f->w_new), "TIMPLE fields");
        die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_W, f->w), "TIMPLE fields");
    }
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_P_OLD, f->p_old), "TIMPLE fields");
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_PPRIME, f->pprime), "TIMPLE fields");
    die_if(mgm_get_field(g_ctx, 0, MGM_FIELD_SOURCE, f->source), "TIMPLE fields");
}

// timple_solver.h:72-175
void calculate_intermediate_velocity_implicit(PointStructure *p, FieldVariables *f)
{
    need_ctx("calculate_intermediate_velocity_implicit");
    timple_params();
    die_if(mgm_timple_part(g_ctx, MGM_TIMPLE_MOMENTUM, g_mode), "calculate_intermediate_velocity_implicit");
    timple_host_view(f, p->num_nodes);
}

// timple_solver.h:177-201
void calculate_mass_residual_implicit(PointStructure *p, FieldVariables *f)
{
    need_ctx("calculate_mass_residual_implicit");
    die_if(mgm_timple_part(g_ctx, MGM_TIMPLE_MASS, g_mode), "calculate_mass_residual_implicit");
    timple_host_view(f, p->num_nodes);
}

// timple_solver.h:341-369
void update_velocity_implicit(PointStructure *p, FieldVariables *f)
{
    need_ctx("update_velocity_implicit");
    die_if(mgm_timple_part(g_ctx, MGM_TIMPLE_UPDATE, g_mode), "update_velocity_implicit");
    timple_host_view(f, p->num_nodes);
}

// timple_solver.h:371-410
void update_boundary_pressure(PointStructure *p, FieldVariables *f)
{
    need_ctx("update_boundary_pressure");
    die_if(mgm_timple_part(g_ctx, MGM_TIMPLE_BOUNDARY_PRESSURE, g_mode), "update_boundary_pressure");
    timple_host_view(f, p->num_nodes);
}

// timple_solver.h:40-70
double time_implicit_solver(PointStructure *ps, FieldVariables *field)
{
    need_ctx("time_implicit_solver");
    timple_params();
    double err = 0;
    die_if(mgm_timple_step(g_ctx, g_mode, &err), "time_implicit_solver");
    // managed-memory view of level 0 (mg_NS_solver.c:75)
    timple_host_view(&field[0], ps[0].num_nodes);
    return err;
}

// ---------------------------------------------------------------------------
// general_functions.h:44-192: the derivative self-test of mg_NS_solver.c:40-43
// (parameters.test > 0).  The manufactured solution and its exact
// derivatives are evaluated on the host with libm, as the reference does
// (pi written 3.14, wave number 1); the operators are applied on the GPU
// (mgm_spmv: the same row sums in the same order as the reference's
// multiply_sparse_matrix_vector); the RMS error over interior nodes is
// summed on the host in node order and printed in the reference's format.
// ---------------------------------------------------------------------------
static double l2_interior(const PointStructure *p, const double *A, const double *B)
{
    double r = 0.0;
    for (int i = 0; i < p->num_nodes; i++)
        if (p->boundary_tag[i] == 0) {
            const double d = A[i] - B[i];
            r += d * d;
        }
    return std::sqrt(r / p->num_nodes);
}

static void apply_op(PointStructure *p, double **D, const double *f, double *out, const char *fn)
{
    const int n = p->num_nodes, k = p->num_cloud_points;
    if (!D || !p->cloud_index) { std::printf("Error: %s: operators not built\n", fn); std::exit(1); }
    std::vector<double> flat = pack_rows(D, n, k);
    std::vector<int> cl = pack_rows(p->cloud_index, n, k);
    die_if(mgm_spmv(n, k, flat.data(), cl.data(), f, out), fn);
}

void test_derivatives(PointStructure *ps, short num_levels, short domain_dimension)
{
    for (int ii = 0; ii < num_levels; ii++) {
        std::printf("Testing level %d\n", ii);
        PointStructure *p = &ps[ii];
        const int n = p->num_nodes;
        const int k = 1;  // wave number
        const bool d3 = domain_dimension > 2;
        std::vector<double> F(n), Fx(n), Fy(n), Fz(n), lapF(n), f(n), fx(n), fy(n), fz(n), lapf(n);
        for (int i = 0; i < n; i++) {
            const double x = p->x[i], y = p->y[i], z = p->z[i];
            if (d3) {
                F[i] = sin(2 * 3.14 * k * x) * sin(2 * 3.14 * k * y) * sin(2 * 3.14 * k * z);
                Fx[i] = 2 * 3.14 * k * cos(2 * 3.14 * k * x) * sin(2 * 3.14 * k * y) * sin(2 * 3.14 * k * z);
                Fy[i] = 2 * 3.14 * k * sin(2 * 3.14 * k * x) * cos(2 * 3.14 * k * y) * sin(2 * 3.14 * k * z);
                Fz[i] = 2 * 3.14 * k * sin(2 * 3.14 * k * x) * sin(2 * 3.14 * k * y) * cos(2 * 3.14 * k * z);
                lapF[i] = -12 * 3.14 * 3.14 * k * k * sin(2 * 3.14 * k * x) * sin(2 * 3.14 * k * y) *
                          sin(2 * 3.14 * k * z);
            } else {
                F[i] = sin(2 * 3.14 * k * x) * sin(2 * 3.14 * k * y);
                Fx[i] = 2 * 3.14 * k * cos(2 * 3.14 * k * x) * sin(2 * 3.14 * k * y);
                Fy[i] = 2 * 3.14 * k * sin(2 * 3.14 * k * x) * cos(2 * 3.14 * k * y);
                lapF[i] = -8 * 3.14 * 3.14 * k * k * sin(2 * 3.14 * k * x) * sin(2 * 3.14 * k * y);
            }
        }
        // the reference overwrites f's derivative slots with the operators applied to f
        f = F;
        apply_op(p, p->Dx, f.data(), fx.data(), "test_derivatives");
        apply_op(p, p->Dy, f.data(), fy.data(), "test_derivatives");
        if (d3) apply_op(p, p->Dz, f.data(), fz.data(), "test_derivatives");
        apply_op(p, p->lap, f.data(), lapf.data(), "test_derivatives");
        const double ef = l2_interior(p, F.data(), f.data()), ex = l2_interior(p, Fx.data(), fx.data()),
                     ey = l2_interior(p, Fy.data(), fy.data()), el = l2_interior(p, lapF.data(), lapf.data());
        if (d3) {
            const double ez = l2_interior(p, Fz.data(), fz.data());
            std::printf("L2 error in f, fx, fy, fz, lapf:\n%lf %lf %lf %lf %lf\n", ef, ex, ey, ez, el);
        } else {
            std::printf("L2 error in f, fx, fy, lapf:\n%lf %lf %lf %lf\n", ef, ex, ey, el);
        }
    }
}

// ---------------------------------------------------------------------------
// structures.h:174-226.  Frees what this library allocated for the levels
// (host arrays and jagged rows; a row array absent on a level, such as
// restr_mat on the finest or prol_mat on the coarsest, is skipped instead of
// being freed row by row as the reference's version does) and releases the
// device context when these are the levels copyin_essentials_to_gpu took.
// ---------------------------------------------------------------------------
static void free_rows(void **rows, int n)
{
    if (!rows) return;
    for (int i = 0; i < n; i++) std::free(rows[i]);
    std::free(rows);
}

void free_PointStructure(PointStructure *ps, int num_levels)
{
    if (!ps) return;
    if (ps == g_ps && g_ctx) {
        mgm_destroy(g_ctx);
        g_ctx = nullptr;
        g_ps = nullptr;
        g_levels = 0;
    }
    for (int l = 0; l < num_levels; l++) {
        PointStructure *p = &ps[l];
        const int n = p->num_nodes;
        void *flat[] = {p->x, p->y, p->z, p->point_index, p->x_normal, p->y_normal, p->z_normal, p->boundary_tag,
                        p->corner_tag, p->pow_x, p->pow_y, p->pow_z, p->prolongation_points, p->restriction_points};
        for (void *a : flat) std::free(a);
        free_rows((void **)p->cloud_index, n);
        free_rows((void **)p->Dx, n);
        free_rows((void **)p->Dy, n);
        free_rows((void **)p->Dz, n);
        free_rows((void **)p->lap, n);
        free_rows((void **)p->lap_Poison, n);
        free_rows((void **)p->restr_mat, n);
        free_rows((void **)p->prol_mat, n);
    }
    std::free(ps);
}

// structures.h:212-226: every member array (the reference's version frees
// only eleven of them)
void free_field(FieldVariables *field, int num_levels)
{
    if (!field) return;
    for (int l = 0; l < num_levels; l++) {
        FieldVariables *f = &field[l];
        double *arrs[] = {f->u, f->v, f->w, f->p, f->u_new, f->v_new, f->w_new, f->u_old, f->v_old, f->w_old,
                          f->p_old, f->pprime, f->res, f->source, f->T, f->dpdn, f->dpdx, f->dpdy, f->dpdz};
        for (double *a : arrs) std::free(a);
    }
    std::free(field);
}

}  // extern "C"
