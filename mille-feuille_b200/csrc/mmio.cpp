// mmio.cpp -- matrix input of the path: Matrix Market (.mtx) and binary CSR
// (.cbd) readers with the reference's semantics (biio2.0/src/biio.h:22-194,
// mmio_highlevel.h:151-323): 1-based -> 0-based, entries placed in file order,
// symmetric / hermitian entries mirrored (diagonal once), pattern -> 1.0,
// integer -> its value, complex -> real part.  The whole file is read at once
// and parsed in memory by all host threads (the reference parses serially
// with fscanf); the result is identical to a serial pass.
#include "../../include/millefeuille.h"

#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <string>
#include <thread>
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

// One chunk of coordinate lines [beg, end), parsed into (row, col, value) in
// file order.  Returns false on a malformed or out-of-range entry.
struct Chunk {
    std::vector<int> ri, ci;
    std::vector<double> vv;
    bool ok = true;
};

void parse_chunk(const char *beg, const char *end, long long M, long long N, bool real, bool complex_,
                 bool integer, Chunk &out)
{
    const char *q = beg;
    char *e = nullptr;
    while (q < end) {
        while (q < end && isspace((unsigned char)*q)) q++;
        if (q >= end) break;
        const long long a = strtoll(q, &e, 10);
        if (e == q) { out.ok = false; return; }
        q = e;
        const long long c = strtoll(q, &e, 10);
        if (e == q) { out.ok = false; return; }
        q = e;
        double v = 1.0;
        if (real || complex_) {
            v = strtod(q, &e);
            if (e == q) { out.ok = false; return; }
            q = e;
            if (complex_) { strtod(q, &e); q = e; }
        } else if (integer) {
            v = (double)(int)strtol(q, &e, 10);
            if (e == q) { out.ok = false; return; }
            q = e;
        }
        if (a < 1 || a > M || c < 1 || c > N) { out.ok = false; return; }
        out.ri.push_back((int)(a - 1));
        out.ci.push_back((int)(c - 1));
        out.vv.push_back(v);
        while (q < end && *q != '\n') q++;     // rest of the line (imaginary part etc.)
    }
}

// Matrix Market coordinate file -> 0-based CSR.  The data lines are cut into
// chunks at line boundaries and parsed by one host thread each; every thread
// then counts its entries per row (mirrored ones included), the per-row
// offsets are the prefix over (row, chunk), and each thread places its entries
// in its own order -- so a row's entries stay in file order, exactly as a
// serial pass places them (a mirrored entry at the position of its line).
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
    while (*q && *q != '\n') q++;               // end of the size line
    const char *data = q, *data_end = buf.data() + buf.size() - 1;

    // chunks at line boundaries, one per thread
    const size_t bytes = (size_t)(data_end - data);
    unsigned hw = std::thread::hardware_concurrency();
    int T = (int)std::min<size_t>(std::max(1u, std::min(hw, 64u)), bytes / (1u << 20) + 1);
    std::vector<const char *> cut(T + 1);
    cut[0] = data;
    cut[T] = data_end;
    for (int k = 1; k < T; k++) {
        const char *c = data + bytes * k / T;
        if (c < cut[k - 1]) c = cut[k - 1];
        while (c < data_end && *c != '\n') c++;
        cut[k] = c;
    }
    std::vector<Chunk> ch(T);
    auto run = [&](auto &&fn) {
        std::vector<std::thread> th;
        for (int k = 1; k < T; k++) th.emplace_back(fn, k);
        fn(0);
        for (auto &x : th) x.join();
    };
    run([&](int k) { parse_chunk(cut[k], cut[k + 1], M, N, real, complex_, integer, ch[k]); });
    long long got = 0;
    for (auto &c : ch) {
        if (!c.ok) return MF_ERR_IO;
        got += (long long)c.ri.size();
    }
    if (got != NZ) return MF_ERR_IO;

    // per-chunk row counts, then offsets in (row, chunk) order
    std::vector<std::vector<int>> cnt(T);
    run([&](int k) {
        cnt[k].assign((size_t)M, 0);
        const Chunk &c = ch[k];
        for (size_t e = 0; e < c.ri.size(); e++) {
            cnt[k][c.ri[e]]++;
            if (sym && c.ri[e] != c.ci[e]) cnt[k][c.ci[e]]++;
        }
    });
    int *rp = (int *)malloc(sizeof(int) * (size_t)(M + 1));
    if (!rp) return MF_ERR_NOMEM;
    long long total = 0;
    for (long long i = 0; i < M; i++) {
        rp[i] = (int)std::min<long long>(total, INT32_MAX);
        for (int k = 0; k < T; k++) {
            const int c = cnt[k][i];
            cnt[k][i] = (int)std::min<long long>(total, INT32_MAX);   // becomes chunk k's cursor in row i
            total += c;
        }
    }
    if (total > INT32_MAX) { free(rp); return MF_ERR_UNSUPPORTED; }
    rp[M] = (int)total;
    int *cc = (int *)malloc(sizeof(int) * (size_t)(total > 0 ? total : 1));
    double *vo = (double *)malloc(sizeof(double) * (size_t)(total > 0 ? total : 1));
    if (!cc || !vo) { free(rp); free(cc); free(vo); return MF_ERR_NOMEM; }
    run([&](int k) {
        const Chunk &c = ch[k];
        std::vector<int> &cur = cnt[k];
        for (size_t e = 0; e < c.ri.size(); e++) {
            int o = cur[c.ri[e]]++;
            cc[o] = c.ci[e];
            vo[o] = c.vv[e];
            if (sym && c.ri[e] != c.ci[e]) {
                o = cur[c.ci[e]]++;
                cc[o] = c.ri[e];
                vo[o] = c.vv[e];
            }
        }
    });
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
