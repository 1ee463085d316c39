// mmio.cpp -- matrix input of the path: Matrix Market (.mtx) and binary CSR
// (.cbd) readers with the reference's semantics (biio2.0/src/biio.h:22-194,
// mmio_highlevel.h:151-323): 1-based -> 0-based, entries placed in file order,
// symmetric / hermitian entries mirrored (diagonal once), pattern -> 1.0,
// integer -> its value, complex -> real part.  The whole file is read at once
// and tokenised in memory (the reference parses with fscanf).
#include "../../include/millefeuille.h"

#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

bool ends_with(const std::string &s, const char *suf)
{
    size_t n = strlen(suf);
    return s.size() >= n && s.compare(s.size() - n, n, suf) == 0;
}

int read_all(const char *path, std::vector<char> &buf)
{
    FILE *f = fopen(path, "rb");
    if (!f) return MF_ERR_IO;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (sz < 0) { fclose(f); return MF_ERR_IO; }
    buf.resize((size_t)sz + 1);
    size_t got = fread(buf.data(), 1, (size_t)sz, f);
    fclose(f);
    if (got != (size_t)sz) return MF_ERR_IO;
    buf[(size_t)sz] = 0;
    return MF_SUCCESS;
}

inline void skip_ws(const char *&p)
{
    while (*p && isspace((unsigned char)*p)) p++;
}

int read_mtx(const char *path, int *m, int *n, int *nnz, int **rowptr, int **colidx, double **val, int *is_sym)
{
    std::vector<char> buf;
    int rc = read_all(path, buf);
    if (rc) return rc;
    char *p = buf.data();
    char *eol = strchr(p, '\n');
    if (!eol) return MF_ERR_IO;
    *eol = 0;
    char t[5][64] = {{0}};
    if (sscanf(p, "%63s %63s %63s %63s %63s", t[0], t[1], t[2], t[3], t[4]) != 5) return MF_ERR_IO;
    for (int k = 1; k < 5; k++)
        for (char *q = t[k]; *q; q++) *q = (char)tolower((unsigned char)*q);
    if (strncmp(t[0], "%%MatrixMarket", 14) != 0 || strcmp(t[1], "matrix") != 0 || strcmp(t[2], "coordinate") != 0)
        return MF_ERR_IO;
    const bool pattern = !strcmp(t[3], "pattern"), real = !strcmp(t[3], "real");
    const bool complex_ = !strcmp(t[3], "complex"), integer = !strcmp(t[3], "integer");
    if (!(pattern || real || complex_ || integer)) return MF_ERR_IO;
    const bool sym = !strcmp(t[4], "symmetric") || !strcmp(t[4], "hermitian");
    const char *q = eol + 1;
    while (*q == '%') {
        const char *e = strchr(q, '\n');
        if (!e) return MF_ERR_IO;
        q = e + 1;
    }
    char *end = nullptr;
    long long M = strtoll(q, &end, 10); q = end;
    long long N = strtoll(q, &end, 10); q = end;
    long long NZ = strtoll(q, &end, 10); q = end;
    if (M <= 0 || N <= 0 || NZ < 0 || M > INT32_MAX || N > INT32_MAX) return MF_ERR_IO;
    std::vector<int> ri((size_t)NZ), ci((size_t)NZ);
    std::vector<double> vv((size_t)NZ);
    std::vector<long long> cnt((size_t)M + 1, 0);
    for (long long k = 0; k < NZ; k++) {
        skip_ws(q);
        long long a = strtoll(q, &end, 10);
        if (end == q) return MF_ERR_IO;
        q = end;
        long long c = strtoll(q, &end, 10);
        if (end == q) return MF_ERR_IO;
        q = end;
        double v = 1.0;
        if (real || complex_) {
            v = strtod(q, &end);
            if (end == q) return MF_ERR_IO;
            q = end;
            if (complex_) { strtod(q, &end); q = end; }
        } else if (integer) {
            v = (double)(int)strtol(q, &end, 10);
            if (end == q) return MF_ERR_IO;
            q = end;
        }
        if (a < 1 || a > M || c < 1 || c > N) return MF_ERR_IO;
        ri[k] = (int)(a - 1);
        ci[k] = (int)(c - 1);
        vv[k] = v;
        cnt[(size_t)(a - 1)]++;
    }
    if (sym)
        for (long long k = 0; k < NZ; k++)
            if (ri[k] != ci[k]) cnt[(size_t)ci[k]]++;
    std::vector<long long> start((size_t)M + 1, 0);
    for (long long i = 0; i < M; i++) start[i + 1] = start[i] + cnt[i];
    const long long total = start[M];
    if (total > INT32_MAX) return MF_ERR_UNSUPPORTED;
    int *rp = (int *)malloc(sizeof(int) * (size_t)(M + 1));
    int *cc = (int *)malloc(sizeof(int) * (size_t)(total > 0 ? total : 1));
    double *vo = (double *)malloc(sizeof(double) * (size_t)(total > 0 ? total : 1));
    if (!rp || !cc || !vo) { free(rp); free(cc); free(vo); return MF_ERR_NOMEM; }
    for (long long i = 0; i <= M; i++) rp[i] = (int)start[i];
    std::vector<long long> fill(start.begin(), start.end() - 1);
    for (long long k = 0; k < NZ; k++) {
        long long o = fill[(size_t)ri[k]]++;
        cc[o] = ci[k];
        vo[o] = vv[k];
        if (sym && ri[k] != ci[k]) {
            o = fill[(size_t)ci[k]]++;
            cc[o] = ri[k];
            vo[o] = vv[k];
        }
    }
    *m = (int)M; *n = (int)N; *nnz = (int)total;
    *rowptr = rp; *colidx = cc; *val = vo; *is_sym = sym ? 1 : 0;
    return MF_SUCCESS;
}

int read_cbd(const char *path, int *m, int *n, int *nnz, int **rowptr, int **colidx, double **val)
{
    FILE *f = fopen(path, "rb");
    if (!f) return MF_ERR_IO;
    int rows = 0, cols = 0;
    int64_t nz = 0;
    int rc = MF_ERR_IO;
    std::vector<int64_t> rp64;
    int *rp = nullptr, *cc = nullptr;
    double *vo = nullptr;
    if (fread(&rows, sizeof(int), 1, f) != 1 || fread(&cols, sizeof(int), 1, f) != 1 ||
        fread(&nz, sizeof(int64_t), 1, f) != 1 || rows < 0 || cols < 0 || nz < 0)
        goto done;
    if (nz > INT32_MAX) { rc = MF_ERR_UNSUPPORTED; goto done; }
    rp64.resize((size_t)rows + 1);
    if (fread(rp64.data(), sizeof(int64_t), (size_t)rows + 1, f) != (size_t)rows + 1) goto done;
    rp = (int *)malloc(sizeof(int) * ((size_t)rows + 1));
    cc = (int *)malloc(sizeof(int) * (size_t)(nz > 0 ? nz : 1));
    vo = (double *)malloc(sizeof(double) * (size_t)(nz > 0 ? nz : 1));
    if (!rp || !cc || !vo) { rc = MF_ERR_NOMEM; goto done; }
    if (fread(cc, sizeof(int), (size_t)nz, f) != (size_t)nz || fread(vo, sizeof(double), (size_t)nz, f) != (size_t)nz)
        goto done;
    for (size_t i = 0; i <= (size_t)rows; i++) rp[i] = (int)rp64[i];
    *m = rows; *n = cols; *nnz = (int)nz;
    *rowptr = rp; *colidx = cc; *val = vo;
    rp = nullptr; cc = nullptr; vo = nullptr;
    rc = MF_SUCCESS;
done:
    fclose(f);
    free(rp); free(cc); free(vo);
    return rc;
}

}  // namespace

extern "C" int mf_read_matrix(const char *path, int *m, int *n, int *nnz, int **rowptr, int **colidx, double **val,
                              int *is_symmetric)
{
    if (!path || !m || !n || !nnz || !rowptr || !colidx || !val) return MF_ERR_INVALID;
    int sym = 0;
    std::string s(path);
    int rc;
    if (ends_with(s, ".cbd")) rc = read_cbd(path, m, n, nnz, rowptr, colidx, val);
    else if (ends_with(s, ".mtx")) rc = read_mtx(path, m, n, nnz, rowptr, colidx, val, &sym);
    else return MF_ERR_IO;
    if (is_symmetric) *is_symmetric = sym;
    return rc;
}

extern "C" int mf_write_cbd(const char *path, int m, int n, int nnz, const int *rowptr, const int *colidx,
                            const double *val)
{
    if (!path || m < 0 || n < 0 || nnz < 0 || !rowptr) return MF_ERR_INVALID;
    FILE *f = fopen(path, "wb");
    if (!f) return MF_ERR_IO;
    int64_t nz = nnz;
    bool ok = fwrite(&m, sizeof(int), 1, f) == 1 && fwrite(&n, sizeof(int), 1, f) == 1 &&
              fwrite(&nz, sizeof(int64_t), 1, f) == 1;
    for (int i = 0; ok && i <= m; i++) {
        int64_t v = rowptr[i];
        ok = fwrite(&v, sizeof(int64_t), 1, f) == 1;
    }
    ok = ok && fwrite(colidx, sizeof(int), (size_t)nnz, f) == (size_t)nnz &&
         fwrite(val, sizeof(double), (size_t)nnz, f) == (size_t)nnz;
    fclose(f);
    return ok ? MF_SUCCESS : MF_ERR_IO;
}
