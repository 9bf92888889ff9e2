/* A C program that drives the library through include/xamg_c_api.h alone, in
 * the order a C user of XAMG's api/c follows (the lifecycle of
 * examples/c/example.c:142-253): init, a CSR matrix filled from host arrays,
 * a partition, vectors uploaded from local vectors, parameters with per-level
 * overrides, a solver, a solve, a parameter change with renew_params, a
 * second solve, the convergence flags, the solution downloaded, everything
 * destroyed, finalize.
 *
 * Test infrastructure: built by tests/test_c_caller.py with the system C
 * compiler as C99 and linked against lib/libxamg_c_api.so. Exit status 0 when
 * every call returned 0 and both solves reached their tolerance (checked
 * here with the true residual of the downloaded solution). */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "xamg_c_api.h"

#define NV 2

#define CHECK(call)                                                         \
    do {                                                                    \
        int rc_ = (call);                                                   \
        if (rc_ != 0) {                                                     \
            fprintf(stderr, "%s returned %d (line %d)\n", #call, rc_, __LINE__); \
            return 1;                                                       \
        }                                                                   \
    } while (0)

/* 7-point Laplacian on an nx*ny*nz grid with Dirichlet boundaries. */
static int build_grid(int nx, int ny, int nz, int **row, int **col, double **val) {
    int n = nx * ny * nz, k = 0;
    *row = malloc((size_t)(n + 1) * sizeof(int));
    *col = malloc((size_t)7 * n * sizeof(int));
    *val = malloc((size_t)7 * n * sizeof(double));
    if (!*row || !*col || !*val) return -1;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) {
                int i = x + nx * (y + ny * z);
                (*row)[i] = k;
                if (z > 0) { (*col)[k] = i - nx * ny; (*val)[k++] = -1.0; }
                if (y > 0) { (*col)[k] = i - nx; (*val)[k++] = -1.0; }
                if (x > 0) { (*col)[k] = i - 1; (*val)[k++] = -1.0; }
                (*col)[k] = i; (*val)[k++] = 6.0;
                if (x < nx - 1) { (*col)[k] = i + 1; (*val)[k++] = -1.0; }
                if (y < ny - 1) { (*col)[k] = i + nx; (*val)[k++] = -1.0; }
                if (z < nz - 1) { (*col)[k] = i + nx * ny; (*val)[k++] = -1.0; }
            }
    (*row)[n] = k;
    return k;
}

/* max over right-hand sides of |b - A x| / |b| */
static double true_rel_res(int n, const int *row, const int *col, const double *val,
                           const double *x, const double *b) {
    double worst = 0.0;
    for (int v = 0; v < NV; ++v) {
        double rr = 0.0, bb = 0.0;
        for (int i = 0; i < n; ++i) {
            double s = b[i * NV + v];
            for (int j = row[i]; j < row[i + 1]; ++j) s -= val[j] * x[col[j] * NV + v];
            rr += s * s;
            bb += b[i * NV + v] * b[i * NV + v];
        }
        double r = sqrt(rr / bb);
        if (r > worst) worst = r;
    }
    return worst;
}

int main(int argc, char **argv) {
    const int nx = 12, ny = 11, nz = 10, n = nx * ny * nz;
    int *row, *col;
    double *val;
    int nnz = build_grid(nx, ny, nz, &row, &col, &val);
    if (nnz < 0) return 1;

    CHECK(XAMG_init(argc, argv, ""));
    if (XAMG_id_get_proc() != 0 || XAMG_id_get_nprocs() != 1) return 1;

    XAMG_vector_id x0, b0;
    CHECK(XAMG_vector_create(&x0, XAMG_MEM_LOCAL));
    CHECK(XAMG_vector_create(&b0, XAMG_MEM_LOCAL));
    CHECK(XAMG_vector_alloc_d(n, NV, x0));
    CHECK(XAMG_vector_alloc_d(n, NV, b0));
    CHECK(XAMG_vector_offset(0, x0));
    CHECK(XAMG_vector_offset(0, b0));
    CHECK(XAMG_vector_set_val_d(0.0, x0));
    double *bh = malloc((size_t)n * NV * sizeof(double));
    double *xh = malloc((size_t)n * NV * sizeof(double));
    for (int i = 0; i < n * NV; ++i) bh[i] = sin(0.37 * i) + 0.25;
    CHECK(XAMG_vector_upload_d(bh, n, 0, NV, b0));

    XAMG_csr_matrix_id csr;
    CHECK(XAMG_csr_matrix_create(&csr));
    CHECK(XAMG_csr_matrix_alloc(n, nnz, csr));
    CHECK(XAMG_csr_matrix_fill(row, col, val, csr));
    CHECK(XAMG_csr_matrix_offset(0, 0, csr));
    if ((int)XAMG_csr_matrix_get_nrows(csr) != n) return 1;

    XAMG_part_id part;
    CHECK(XAMG_part_create(&part));
    CHECK(XAMG_part_construct(n, part));
    XAMG_matrix_id m;
    CHECK(XAMG_matrix_create(&m));
    CHECK(XAMG_matrix_set_part(part, m));
    CHECK(XAMG_matrix_construct(csr, m));
    CHECK(XAMG_csr_matrix_destroy(csr));

    XAMG_param_id par;
    CHECK(XAMG_param_create(&par));
    CHECK(XAMG_param_add_value_s("solver", "method", "PBiCGStab", par));
    CHECK(XAMG_param_add_value_d("solver", "rel_tolerance", 1.e-6f, par));
    CHECK(XAMG_param_add_value_d("solver", "abs_tolerance", 0.0f, par));
    CHECK(XAMG_param_add_value_s("preconditioner", "method", "MultiGrid", par));
    CHECK(XAMG_param_add_value_i("preconditioner", "mg_coarse_matrix_size", 50, par));
    /* the host setup implements PMIS (8) with extended+i (6), no aggressive levels */
    CHECK(XAMG_param_add_value_i("preconditioner", "mg_coarsening_type", 8, par));
    CHECK(XAMG_param_add_value_i("preconditioner", "mg_interpolation_type", 6, par));
    CHECK(XAMG_param_add_value_i("preconditioner", "mg_agg_num_levels", 0, par));
    /* out-of-range values are refused (polynomial_order is 1..4) */
    if (XAMG_param_add_value_i("pre_smoother", "polynomial_order", 9, par) == 0) return 3;
    XAMG_param_override_id ov;
    CHECK(XAMG_param_override_create(&ov));
    CHECK(XAMG_param_override_add_value("mg_coarsening_type", "8@lev0-1", ov));
    CHECK(XAMG_param_override_add_value("mg_interpolation_type", "6@lev0-1", ov));
    CHECK(XAMG_param_override_apply("preconditioner", par, ov));
    CHECK(XAMG_param_override_destroy(ov));
    XAMG_param_set_default(par);

    XAMG_vector_id x, b;
    CHECK(XAMG_vector_create(&x, XAMG_MEM_DISTRIBUTED));
    CHECK(XAMG_vector_create(&b, XAMG_MEM_DISTRIBUTED));
    CHECK(XAMG_vector_set_part(part, x));
    CHECK(XAMG_vector_set_part(part, b));
    int local = XAMG_part_get_numa_size(part);
    if (local != n) return 1;
    CHECK(XAMG_vector_alloc_d(local, NV, x));
    CHECK(XAMG_vector_alloc_d(local, NV, b));
    CHECK(XAMG_vector_upload_v(x0, x));
    CHECK(XAMG_vector_upload_v(b0, b));

    XAMG_solver_id sol;
    CHECK(XAMG_solver_create2(m, par, x, b, &sol));
    CHECK(XAMG_barrier());
    double t0 = XAMG_timer();
    CHECK(XAMG_solver_solve1(NV, sol));
    double t1 = XAMG_timer();
    CHECK(XAMG_vector_download_d(xh, n, 0, NV, x));
    double r1 = true_rel_res(n, row, col, val, xh, bh);

    /* tighter tolerance, new parameters, solve again from zero */
    CHECK(XAMG_param_change_value_d("solver", "rel_tolerance", 1.e-8f, par));
    CHECK(XAMG_solver_renew_params(par, sol));
    CHECK(XAMG_vector_upload_v(x0, x));
    CHECK(XAMG_solver_solve1(NV, sol));
    int conv[NV];
    CHECK(XAMG_solver_get_convergence_info(conv, NV, sol));
    CHECK(XAMG_vector_download_d(xh, n, 0, NV, x));
    double r2 = true_rel_res(n, row, col, val, xh, bh);

    CHECK(XAMG_vector_destroy(x));
    CHECK(XAMG_vector_destroy(b));
    CHECK(XAMG_vector_destroy(x0));
    CHECK(XAMG_vector_destroy(b0));
    CHECK(XAMG_solver_destroy(sol));
    CHECK(XAMG_matrix_destroy(m));
    CHECK(XAMG_part_destroy(part));
    CHECK(XAMG_param_destroy(par));
    CHECK(XAMG_finalize());

    printf("lifecycle: n=%d nnz=%d first solve %.3f ms rel_res %.3e, second rel_res %.3e, "
           "conv %d %d\n", n, nnz, (t1 - t0) * 1e3, r1, r2, conv[0], conv[1]);
    free(row);
    free(col);
    free(val);
    free(bh);
    free(xh);
    return (r1 <= 1e-5 && r2 <= 1e-7 && conv[0] && conv[1]) ? 0 : 2;
}
