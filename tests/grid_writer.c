/*
 * grid_writer.c -- calls the write_functions.h writers of libmgm.so
 * (include/mgm_reference.h) on a level read from a binary file, for
 * tests/test_writers.py.
 *
 *   grid_writer <level.bin> <level>      write_processed_grid_data into the cwd
 *   grid_writer <arrays.bin> test <dir/> write_test_files with prefix dir/
 *
 * level.bin: int32 n, k; double x, y, z, nx, ny, nz [n]; uint8 btag, corner [n];
 *            int32 cloud [n][k], ppts [n], rpts [n].
 * arrays.bin: int32 n; double f, fx, fy, fz, lapf, fxx, fyy, fzz [n].
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mgm_reference.h"

static void rd(void *p, size_t sz, size_t n, FILE *f)
{
    if (fread(p, sz, n, f) != n) { fprintf(stderr, "short read\n"); exit(2); }
}

int main(int argc, char **argv)
{
    if (argc < 3) return 1;
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 1;
    if (strcmp(argv[2], "test") == 0) {
        int n;
        rd(&n, sizeof(int), 1, f);
        double *a[8];
        for (int t = 0; t < 8; t++) { a[t] = malloc(sizeof(double) * n); rd(a[t], sizeof(double), n, f); }
        write_test_files(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], n, argv[3]);
        return 0;
    }
    int hdr[2];
    rd(hdr, sizeof(int), 2, f);
    const int n = hdr[0], k = hdr[1];
    PointStructure p;
    memset(&p, 0, sizeof(p));
    AllocateMemoryPointStructure(&p, n);
    p.num_cloud_points = (short)k;
    double *d[6] = {p.x, p.y, p.z, p.x_normal, p.y_normal, p.z_normal};
    for (int t = 0; t < 6; t++) rd(d[t], sizeof(double), n, f);
    unsigned char *bt = malloc(n), *ct = malloc(n);
    rd(bt, 1, n, f);
    rd(ct, 1, n, f);
    for (int i = 0; i < n; i++) { p.boundary_tag[i] = bt[i] != 0; p.corner_tag[i] = ct[i] != 0; }
    p.cloud_index = malloc(sizeof(int *) * n);
    for (int i = 0; i < n; i++) { p.cloud_index[i] = malloc(sizeof(int) * k); rd(p.cloud_index[i], sizeof(int), k, f); }
    p.prolongation_points = malloc(sizeof(int) * n);
    p.restriction_points = malloc(sizeof(int) * n);
    rd(p.prolongation_points, sizeof(int), n, f);
    rd(p.restriction_points, sizeof(int), n, f);
    fclose(f);
    write_processed_grid_data(&p, atoi(argv[2]));
    return 0;
}
