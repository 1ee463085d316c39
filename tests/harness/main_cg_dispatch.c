/*
 * A program written against the reference's main-cg entry points, as a user
 * of the reference would link it: the dispatch of main-cg.cu:1727-1745 (nnz <
 * 10,000 -> cg_solve_inc, < 100,000 -> cg_solve_sync, else cg_solve_reduce)
 * on b = A x with x = 1 (Y_golden, main-cg.cu:1715-1720), a fixed iteration
 * count, then the library's record of the last drop-in solve.
 *
 *   main_cg_dispatch matrix.mtx max_iter
 *
 * Prints one line: entry=<name> iterations=<n> l2_norm=<v> tiles=<fp64>,<fp32>,<fp16>,<int8>
 * Built and run by tests/test_gpu_dropin_dispatch.py against libmillefeuille.so
 * and libmillefeuille_fp64.so.
 */
#include <stdio.h>
#include <stdlib.h>

#include "millefeuille.h"

int main(int argc, char **argv)
{
    if (argc < 3) {
        fprintf(stderr, "usage: main_cg_dispatch matrix.mtx max_iter\n");
        return 1;
    }
    int m = 0, n = 0, nnz = 0, sym = 0;
    int *rowptr = NULL, *colidx = NULL;
    double *val = NULL;
    if (mf_read_matrix(argv[1], &m, &n, &nnz, &rowptr, &colidx, &val, &sym) != 0) return 2;
    const int max_iter = atoi(argv[2]);
    const int rows = (m / 16) * 16;
    float *val_low = (float *)malloc(sizeof(float) * (size_t)(nnz > 0 ? nnz : 1));
    double *x = (double *)calloc((size_t)n, sizeof(double));
    double *b = (double *)calloc((size_t)n, sizeof(double));
    for (int i = 0; i < nnz; i++) val_low[i] = (float)val[i];
    for (int i = 0; i < rows; i++)
        for (int j = rowptr[i]; j < rowptr[i + 1]; j++) b[i] += val[j];
    int iter = 0;
    CgBenchResult res;
    const char *entry;
    if (nnz < 10000) {
        entry = "cg_solve_inc";
        cg_solve_inc(rowptr, colidx, val, val_low, x, b, rows, &iter, 10, 1e-5, argv[1], nnz, n, max_iter, &res, 1);
    } else if (nnz < 100000) {
        entry = "cg_solve_sync";
        cg_solve_sync(rowptr, colidx, val, val_low, x, b, rows, &iter, 10, 1e-5, argv[1], nnz, n, max_iter, &res, 1);
    } else {
        entry = "cg_solve_reduce";
        cg_solve_reduce(rowptr, colidx, val, val_low, x, b, rows, &iter, 10, 1e-5, argv[1], nnz, n, max_iter, &res, 1);
    }
    mf_report rep;
    if (mf_dropin_last_report(&rep) != 0) return 3;
    printf("entry=%s iterations=%d l2_norm=%.17g tiles=%lld,%lld,%lld,%lld arch=%s\n", entry, res.iterations,
           res.l2_norm, rep.tile_uses[0], rep.tile_uses[1], rep.tile_uses[2], rep.tile_uses[3], mf_build_arch());
    mf_free_host(rowptr);
    mf_free_host(colidx);
    mf_free_host(val);
    free(val_low);
    free(x);
    free(b);
    return 0;
}
