// driver_main.cpp -- the reference's four benchmark executables, as drop-in
// programs over libmillefeuille.so (same command lines, prints and CSV rows,
// so test_Mille_feuille.sh runs them unchanged):
//
//   main-cg         <matrix> <max_iter> [out.csv]   FP64 CG        (main-cg.cu:1682-1764)
//   main-cg-mixed   <matrix> <max_iter> [out.csv]   mixed CG       (main-cg-mixed.cu:3071-3144)
//   main-bicg       <matrix>                        FP64 BiCGSTAB  (main-bicg.cu main)
//   main-bicg-mixed <matrix>                        mixed BiCGSTAB (main-bicg-mixed.cu:2168-2193)
//
// The variant is chosen at compile time (MF_DRIVER 0..3).  As in the
// reference: the matrix is read with read_Dmatrix_32's semantics, rows and
// columns are truncated to a multiple of 16, b = A 1, the CG solve runs 3
// warm-up and 10 timed calls with exactly max_iter iterations, and one row
// "matrix,variant,iterations,time_ms,nnz,l2_norm,residual" is appended to the
// CSV (header when the file is empty).  BiCGSTAB: rhs = 1, x = 0, one call;
// the entry point prints and appends its own row.  Differences: a missing
// argument prints the usage instead of crashing, and the CSV columns hold the
// solver's reported iterations and FP64 true residual.
#include "../../include/millefeuille.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#ifndef MF_DRIVER
#define MF_DRIVER 1
#endif

namespace {
constexpr int kWarmup = 3;
constexpr int kBenchmark = 10;
constexpr int kBlock = 16;

const char *kName[] = {"main-cg", "main-cg-mixed", "main-bicg", "main-bicg-mixed"};

int run_cg(const char *filename, int max_iter, const char *out_csv)
{
    int m, n, nnz, sym;
    int *rowptr = nullptr, *colidx = nullptr;
    double *val = nullptr;
    int rc = mf_read_matrix(filename, &m, &n, &nnz, &rowptr, &colidx, &val, &sym);
    if (rc != MF_SUCCESS) {
        fprintf(stderr, "%s: cannot read %s: %s\n", kName[MF_DRIVER], filename, mf_status_string(rc));
        return 1;
    }
    if (m != n) {
        printf("unequal\n");
        return 0;
    }
    printf("matrix rows=%d cols=%d nnz=%d\n", m, n, nnz);
    std::vector<float> val_low(nnz > 0 ? nnz : 1);
    for (int i = 0; i < nnz; i++) val_low[i] = (float)val[i];
    const int ori = n;
    n = (n / kBlock) * kBlock;
    std::vector<double> x(n > 0 ? n : 1, 0.0), b(n > 0 ? n : 1, 0.0);
    for (int i = 0; i < n; i++)          // b = A 1 over the kept rows
        for (int j = rowptr[i]; j < rowptr[i + 1]; j++) b[i] += val[j];
    int iter = 0;
    CgBenchResult result = {0.0, 0, 0.0, 0.0};
    auto solve = [&](CgBenchResult *res) {
        if (MF_DRIVER == 0)
            cg_solve_sync(rowptr, colidx, val, val_low.data(), x.data(), b.data(), n, &iter, 10, 1e-5,
                          (char *)filename, nnz, ori, max_iter, res, 1);
        else
            cg_solve_inc(rowptr, colidx, val, val_low.data(), x.data(), b.data(), n, &iter, 10, 1e-5,
                         (char *)filename, nnz, ori, max_iter, res, 1);
    };
    for (int i = 0; i < kWarmup; i++) solve(nullptr);
    double avg = 0.0;
    for (int i = 0; i < kBenchmark; i++) {
        solve(&result);
        avg += result.time_ms;
    }
    avg /= kBenchmark;
    printf("%s=%.3f ms (warmup=%d, benchmark=%d)\n", MF_DRIVER == 0 ? "time_cg_avg" : "time_cg-mixed_avg", avg,
           kWarmup, kBenchmark);
    FILE *f = fopen(out_csv, "a");
    if (f) {
        if (ftell(f) == 0) fprintf(f, "matrix,variant,iterations,time_ms,nnz,l2_norm,residual\n");
        fprintf(f, "%s,%s,%d,%.3f,%d,%e,%e\n", filename, MF_DRIVER == 0 ? "cg" : "cg_mixed", result.iterations, avg,
                nnz, result.l2_norm, result.residual);
        fclose(f);
    }
    mf_free_host(rowptr);
    mf_free_host(colidx);
    mf_free_host(val);
    return 0;
}

int run_bicg(const char *filename)
{
    int m, n, nnz, sym;
    int *rowptr = nullptr, *colidx = nullptr;
    double *val = nullptr;
    int rc = mf_read_matrix(filename, &m, &n, &nnz, &rowptr, &colidx, &val, &sym);
    if (rc != MF_SUCCESS) {
        fprintf(stderr, "%s: cannot read %s: %s\n", kName[MF_DRIVER], filename, mf_status_string(rc));
        return 1;
    }
    std::vector<double> x(m > 0 ? m : 1, 0.0), rhs(m > 0 ? m : 1, 1.0);
    if (MF_DRIVER == 3) bicgstab(rowptr, colidx, val, rhs.data(), x.data(), nnz, (char *)filename, m);
    else bicgstab_sync(rowptr, colidx, val, rhs.data(), x.data(), nnz, (char *)filename, m);
    mf_free_host(rowptr);
    mf_free_host(colidx);
    mf_free_host(val);
    return 0;
}
}  // namespace

int main(int argc, char **argv)
{
    const bool cg = MF_DRIVER < 2;
    if (argc < (cg ? 3 : 2)) {
        fprintf(stderr, cg ? "usage: %s <matrix.mtx|.cbd> <max_iter> [out.csv]\n" : "usage: %s <matrix.mtx|.cbd>\n",
                kName[MF_DRIVER]);
        return 1;
    }
    if (cg) {
        const char *csv = argc >= 4 ? argv[3] : (MF_DRIVER == 0 ? "cg_performance.csv" : "cg_mixed_performance.csv");
        return run_cg(argv[1], atoi(argv[2]), csv);
    }
    return run_bicg(argv[1]);
}
