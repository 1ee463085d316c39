/*
 * mf_oracle.c -- CPU restatement of Mille-feuille's tile path.
 *
 * TEST INFRASTRUCTURE ONLY (the test oracle).  Only tests/, smoke() and bench.py's
 * cpu_baseline / reference arm call this code.  The product never does.
 *
 * Each function names the reference file:line (inside the zhaijiaqi/Mille-feuille
 * project, under src/) whose behaviour it restates.  The code is written
 * from the behaviour, not copied: the reference's O(tilem * tilen) per-tile-row
 * scratch arrays are replaced by a stamp array so the same output is produced
 * in O(nnz log) time (the reference cannot tile the 128^3 system in reasonable
 * time on a host).
 */
#include "mf_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <ctype.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define BS 16

static size_t vec_len(const orc_tiles *T, int n);
static void spmv_tile_exact(const orc_tiles *T, int rowA, const double *x, double *y, int nthreads);

void orc_free(void *p) { free(p); }

static int cmp_int(const void *a, const void *b)
{
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

/* exclusive_scan (utils.h:34-49): out[0]=0, out[i]=in[i-1]+out[i-1]. */
static void xscan_int(int *a, int len)
{
    if (len <= 1) return;
    int prev = a[0];
    a[0] = 0;
    for (int i = 1; i < len; i++) {
        int cur = a[i];
        a[i] = prev + a[i - 1];
        prev = cur;
    }
}

/* exclusive_scan_char (utils.h:50-64): the same scan in uint8 arithmetic. */
static void xscan_u8(unsigned char *a, int len)
{
    if (len <= 1) return;
    unsigned char prev = a[0];
    a[0] = 0;
    for (int i = 1; i < len; i++) {
        unsigned char cur = a[i];
        a[i] = (unsigned char)(prev + a[i - 1]);
        prev = cur;
    }
}

void orc_tiles_free(orc_tiles *T)
{
    free(T->tile_ptr); free(T->tile_columnidx); free(T->tile_nnz); free(T->blknnz);
    free(T->csr_offset); free(T->csrptr_offset); free(T->val); free(T->val_low);
    free(T->col); free(T->ptr);
    memset(T, 0, sizeof(*T));
}

/*
 * Tile_create (csr2block.h:267-422) with convert_step1..4 (csr2block.h:6-265).
 *  - tile-row R covers rows [16R, min(16R+16, rowA)); its entries are
 *    rowptr[16R] .. rowptr[end) (csr2block.h:28-30).
 *  - tiles of a tile-row are the distinct column tiles, ascending (step 2,
 *    csr2block.h:89-102).
 *  - per-(tile,row) counts are uint8 and scanned in uint8 (csr2block.h:85,237).
 *  - payload: entries of a tile in CSR order, then copied row by row with the
 *    uint8 row starts (csr2block.h:204-253).
 *  - tile_nnz, blknnz, csr_offset are the same exclusive scan of tile nnz;
 *    csrptr_offset is the exclusive scan of the tile-row height
 *    (csr2block.h:144-147,319,346-347,376).
 */
int orc_tile_create(int rowA, int colA, const int *rowptr, const int *colidx,
                    const double *val, const float *val_low, orc_tiles *T)
{
    memset(T, 0, sizeof(*T));
    if (rowA < 0 || colA < 0) return -1;
    const int tilem = (rowA + BS - 1) / BS;
    const int tilen = (colA + BS - 1) / BS;
    T->tilem = tilem;
    T->tilen = tilen;
    T->tile_ptr = (int *)calloc((size_t)tilem + 1, sizeof(int));
    int *stamp = (int *)malloc(((size_t)tilen + 1) * sizeof(int));
    int *pos = (int *)malloc(((size_t)tilen + 1) * sizeof(int));
    for (int j = 0; j < tilen; j++) stamp[j] = -1;

    /* step 1: distinct column tiles per tile-row (csr2block.h:22-39). */
    for (int R = 0; R < tilem; R++) {
        int start = R * BS, end = (R == tilem - 1) ? rowA : (R + 1) * BS;
        int cnt = 0;
        for (int j = rowptr[start]; j < rowptr[end]; j++) {
            int jc = colidx[j] / BS;
            if (stamp[jc] != R) { stamp[jc] = R; cnt++; }
        }
        T->tile_ptr[R] = cnt;
    }
    xscan_int(T->tile_ptr, tilem + 1);
    const int tilenum = T->tile_ptr[tilem];
    T->tilenum = tilenum;
    T->tile_columnidx = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    T->tile_nnz = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    T->blknnz = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    T->csr_offset = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    T->csrptr_offset = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    unsigned char *tcp = (unsigned char *)calloc((size_t)tilenum * BS + 1, 1);

    /* step 2: column ids, tile nnz, per-(tile,row) uint8 counts. */
    for (int j = 0; j < tilen; j++) stamp[j] = -1;
    int *list = (int *)malloc(((size_t)tilen + 1) * sizeof(int));
    for (int R = 0; R < tilem; R++) {
        int start = R * BS, end = (R == tilem - 1) ? rowA : (R + 1) * BS;
        int rowlen = end - start;
        int cnt = 0;
        for (int j = rowptr[start]; j < rowptr[end]; j++) {
            int jc = colidx[j] / BS;
            if (stamp[jc] != R) { stamp[jc] = R; list[cnt++] = jc; }
        }
        qsort(list, (size_t)cnt, sizeof(int), cmp_int);
        int t0 = T->tile_ptr[R];
        for (int s = 0; s < cnt; s++) {
            T->tile_columnidx[t0 + s] = list[s];
            pos[list[s]] = s;
        }
        for (int ri = 0; ri < rowlen; ri++)
            for (int j = rowptr[start + ri]; j < rowptr[start + ri + 1]; j++) {
                int t = t0 + pos[colidx[j] / BS];
                T->tile_nnz[t]++;
                tcp[(size_t)t * BS + ri]++;
            }
        /* step 3 (csr2block.h:131-149): blknnz, csr_offset = nnz; csrptr_offset = rowlen */
        for (int s = 0; s < cnt; s++) {
            T->blknnz[t0 + s] = T->tile_nnz[t0 + s];
            T->csr_offset[t0 + s] = T->tile_nnz[t0 + s];
            T->csrptr_offset[t0 + s] = rowlen;
        }
    }
    xscan_int(T->tile_nnz, tilenum + 1);
    xscan_int(T->csr_offset, tilenum + 1);
    xscan_int(T->csrptr_offset, tilenum + 1);
    /* csrsize / csrptrlen (csr2block.h:349-371) */
    long long csrsize = 0, csrptrlen = 0;
    for (int t = 0; t < tilenum; t++) {
        csrsize += T->blknnz[t];
        csrptrlen += T->csrptr_offset[t + 1] - T->csrptr_offset[t];
    }
    xscan_int(T->blknnz, tilenum + 1);
    T->csrsize = (int)csrsize;
    T->csrptrlen = (int)csrptrlen;
    T->val = (double *)calloc((size_t)csrsize + 1, sizeof(double));
    T->val_low = (float *)calloc((size_t)csrsize + 1, sizeof(float));
    T->col = (unsigned char *)calloc((size_t)csrsize + 1, 1);
    T->ptr = (unsigned char *)calloc((size_t)csrptrlen + 1, 1);

    /* step 4 (csr2block.h:187-260): per tile-row temp payload in CSR order,
     * then copied row by row using the uint8 row starts. */
    int maxrow_nnz = 0;
    for (int R = 0; R < tilem; R++) {
        int start = R * BS, end = (R == tilem - 1) ? rowA : (R + 1) * BS;
        int c = rowptr[end] - rowptr[start];
        if (c > maxrow_nnz) maxrow_nnz = c;
    }
    double *tv = (double *)malloc(((size_t)maxrow_nnz + 1) * sizeof(double));
    float *tvl = (float *)malloc(((size_t)maxrow_nnz + 1) * sizeof(float));
    unsigned char *tc = (unsigned char *)malloc((size_t)maxrow_nnz + 1);
    int *cursor = (int *)malloc(((size_t)tilen + 1) * sizeof(int));
    for (int j = 0; j < tilen; j++) stamp[j] = -1;
    for (int R = 0; R < tilem; R++) {
        int start = R * BS, end = (R == tilem - 1) ? rowA : (R + 1) * BS;
        int rowlen = end - start;
        int t0 = T->tile_ptr[R], t1 = T->tile_ptr[R + 1];
        for (int t = t0; t < t1; t++) {
            pos[T->tile_columnidx[t]] = t - t0;
            cursor[t - t0] = 0;
        }
        for (int j = rowptr[start]; j < rowptr[end]; j++) {
            int jc = colidx[j] / BS;
            int s = pos[jc];
            int pre = T->tile_nnz[t0 + s] - T->tile_nnz[t0];
            int k = pre + cursor[s]++;
            tv[k] = val[j];
            tvl[k] = val_low[j];
            tc[k] = (unsigned char)(colidx[j] - jc * BS);
        }
        for (int t = t0; t < t1; t++) {
            int pre = T->tile_nnz[t] - T->tile_nnz[t0];
            int nnzt = T->tile_nnz[t + 1] - T->tile_nnz[t];
            int off = T->csr_offset[t], poff = T->csrptr_offset[t];
            unsigned char *pt = tcp + (size_t)t * BS;
            xscan_u8(pt, rowlen);
            for (int ri = 0; ri < rowlen; ri++) {
                int st = pt[ri];
                int sp = (ri == rowlen - 1) ? nnzt : pt[ri + 1];
                for (int k = st; k < sp; k++) {
                    T->val[off + k] = tv[pre + k];
                    T->val_low[off + k] = tvl[pre + k];
                    T->col[off + k] = tc[pre + k];
                }
                T->ptr[poff + ri] = pt[ri];
            }
        }
    }
    free(tv); free(tvl); free(tc); free(cursor); free(list); free(stamp); free(pos); free(tcp);
    return 0;
}

/* blockspmv_cpu (blockspmv_cpu.h:2-112): row-block split with PREFETCH_SMEM_TH=4
 * (common.h:61) and the per-tile value / row-pointer offsets. */
int orc_offsets_build(const orc_tiles *T, int rowA, orc_offsets *O)
{
    memset(O, 0, sizeof(*O));
    const int tilem = T->tilem, TH = 4;
    int rb = 0;
    for (int R = 0; R < tilem; R++) {
        int nb = T->tile_ptr[R + 1] - T->tile_ptr[R];
        rb += (nb <= TH) ? 1 : (int)ceil((double)nb / (double)TH);
    }
    O->rowblkblock = rb;
    O->blkcoostylerowidx = (unsigned int *)calloc((size_t)rb + 1, sizeof(unsigned int));
    O->colstart = (int *)calloc((size_t)rb + 1, sizeof(int));
    O->colstop = (int *)calloc((size_t)rb + 1, sizeof(int));
    int c = 0;
    for (int R = 0; R < tilem; R++) {
        int nb = T->tile_ptr[R + 1] - T->tile_ptr[R];
        if (nb <= TH) {
            O->blkcoostylerowidx[c++] = (unsigned int)R;
        } else {
            int num = (int)ceil((double)nb / (double)TH);
            int len = (int)ceil((double)nb / (double)num);
            for (int i = 0; i < num; i++) {
                O->blkcoostylerowidx[c] = (unsigned int)R | 0x80000000u;
                O->colstart[c] = T->tile_ptr[R] + i * len;
                O->colstop[c] = (i == num - 1) ? T->tile_ptr[R] + nb : T->tile_ptr[R] + (i + 1) * len;
                c++;
            }
        }
    }
    O->ptroffset1 = (int *)calloc((size_t)T->tilenum + 1, sizeof(int));
    O->ptroffset2 = (int *)calloc((size_t)T->tilenum + 1, sizeof(int));
    int vo = 0, po = 0;
    for (int R = 0; R < tilem; R++) {
        int rowlen = (R == tilem - 1) ? rowA - (tilem - 1) * BS : BS;
        for (int t = T->tile_ptr[R]; t < T->tile_ptr[R + 1]; t++) {
            O->ptroffset1[t] = vo;
            O->ptroffset2[t] = po;
            vo += T->blknnz[t + 1] - T->blknnz[t];
            po += rowlen;
        }
    }
    return 0;
}

void orc_offsets_free(orc_offsets *O)
{
    free(O->ptroffset1); free(O->ptroffset2); free(O->blkcoostylerowidx);
    free(O->colstart); free(O->colstop);
    memset(O, 0, sizeof(*O));
}

/* Nonempty-row lists (main-cg-mixed.cu:2447-2514), single-thread semantics.
 * (The reference's first loop shares `csrcount` across OpenMP threads, a data
 * race; the deterministic result is the serial one restated here.) */
int orc_rowlists_build(const orc_tiles *T, int rowA, orc_rowlists *L)
{
    memset(L, 0, sizeof(*L));
    const int tilem = T->tilem, tilenum = T->tilenum;
    L->nonzero_row_new = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    L->tile_rowidx = (int *)calloc((size_t)tilenum + 1, sizeof(int));
    L->block_signal = (int *)calloc((size_t)tilem + 4, sizeof(int));
    for (int R = 0; R < tilem; R++) {
        int rowlen = (R == tilem - 1) ? rowA - (tilem - 1) * BS : BS;
        for (int t = T->tile_ptr[R]; t < T->tile_ptr[R + 1]; t++) {
            int cc = T->csrptr_offset[t];
            L->tile_rowidx[t] = R;
            int cnt = 0;
            for (int ri = 0; ri < rowlen; ri++) {
                int stop = (ri == rowlen - 1) ? (T->blknnz[t + 1] - T->blknnz[t]) : T->ptr[ri + 1 + cc];
                if (stop != T->ptr[cc + ri]) cnt++;
            }
            L->nonzero_row_new[t] = cnt + 1;
        }
    }
    xscan_int(L->nonzero_row_new, tilenum + 1);
    L->cnt = L->nonzero_row_new[tilenum];
    L->blockrowid_new = (unsigned char *)calloc((size_t)L->cnt + 1, 1);
    L->blockcsr_ptr_new = (unsigned char *)calloc((size_t)L->cnt + 1, 1);
    for (int R = 0; R < tilem; R++) {
        int rowlen = (R == tilem - 1) ? rowA - (tilem - 1) * BS : BS;
        L->block_signal[R] = T->tile_ptr[R + 1] - T->tile_ptr[R];
        for (int t = T->tile_ptr[R]; t < T->tile_ptr[R + 1]; t++) {
            int cc = T->csrptr_offset[t];
            int base = L->nonzero_row_new[t];
            int fl = 0;
            for (int ri = 0; ri < rowlen; ri++) {
                int stop = (ri == rowlen - 1) ? (T->blknnz[t + 1] - T->blknnz[t]) : T->ptr[ri + 1 + cc];
                if (ri == 0) {
                    L->blockrowid_new[base + fl] = 0;
                    L->blockcsr_ptr_new[base + fl] = 0;
                    fl++;
                }
                if (stop != T->ptr[cc + ri]) {
                    L->blockrowid_new[base + fl] = (unsigned char)ri;
                    L->blockcsr_ptr_new[base + fl] = (unsigned char)stop;
                    fl++;
                }
            }
        }
    }
    return 0;
}

void orc_rowlists_free(orc_rowlists *L)
{
    free(L->nonzero_row_new); free(L->blockrowid_new); free(L->blockcsr_ptr_new);
    free(L->tile_rowidx); free(L->block_signal);
    memset(L, 0, sizeof(*L));
}

/* IEEE binary32 -> binary16, round to nearest, ties to even (the host
 * conversion the reference's `(half)float` performs, main-cg-mixed.cu:2344).
 * Written from the IEEE 754 definition. */
uint16_t orc_f32_to_f16_rn(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    uint32_t sign = (u >> 16) & 0x8000u;
    uint32_t ex = (u >> 23) & 0xFFu;
    uint32_t man = u & 0x7FFFFFu;
    if (ex == 0xFFu) {                         /* inf / nan */
        if (man == 0) return (uint16_t)(sign | 0x7C00u);
        return (uint16_t)(sign | 0x7E00u | (man >> 13));
    }
    int e = (int)ex - 127 + 15;                /* rebias */
    if (e >= 31) return (uint16_t)(sign | 0x7C00u);   /* overflow -> inf */
    if (e <= 0) {                              /* subnormal or zero in half */
        if (e < -10) return (uint16_t)sign;    /* below half of min subnormal */
        uint32_t m = man | 0x800000u;          /* implicit bit */
        int shift = 14 - e;                    /* bits to drop: 13 + (1 - e) */
        uint32_t q = m >> shift;
        uint32_t rem = m & ((1u << shift) - 1u);
        uint32_t half = 1u << (shift - 1);
        if (rem > half || (rem == half && (q & 1u))) q++;
        return (uint16_t)(sign | q);
    }
    uint32_t q = ((uint32_t)e << 10) | (man >> 13);
    uint32_t rem = man & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (q & 1u))) q++;  /* may carry into exponent: correct */
    return (uint16_t)(sign | q);
}

float orc_f16_to_f32(uint16_t h)
{
    uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
    uint32_t ex = (h >> 10) & 0x1Fu;
    uint32_t man = h & 0x3FFu;
    uint32_t u;
    if (ex == 0) {
        if (man == 0) u = sign;
        else {                                  /* normalise the subnormal */
            int e = -1;
            do { man <<= 1; e++; } while (!(man & 0x400u));
            man &= 0x3FFu;
            u = sign | ((uint32_t)(127 - 15 - e) << 23) | (man << 13);
        }
    } else if (ex == 0x1F) {
        u = sign | 0x7F800000u | (man << 13);
    } else {
        u = sign | ((ex - 15 + 127) << 23) | (man << 13);
    }
    float f;
    memcpy(&f, &u, 4);
    return f;
}

/* binary64 -> binary16, round to nearest even, of the exact value s + e where
 * |e| is below half an ulp of s (TwoSum's error term; 0 for a plain double).
 * Written from the IEEE 754 definition: the dropped bits of s decide the
 * rounding, and only when they sit exactly on the halfway point does e (its
 * sign relative to s) break the tie; e = 0 breaks it to even. */
uint16_t orc_f64_to_f16_rn(double s, double e)
{
    uint64_t u;
    memcpy(&u, &s, 8);
    uint16_t sign = (uint16_t)((u >> 48) & 0x8000u);
    int ex = (int)((u >> 52) & 0x7FF);
    uint64_t man = u & 0xFFFFFFFFFFFFFull;
    if (ex == 0x7FF) {                          /* inf / nan */
        if (man == 0) return (uint16_t)(sign | 0x7C00u);
        return (uint16_t)(sign | 0x7E00u | (uint16_t)(man >> 42));
    }
    if (ex == 0) return sign;                   /* zero or double subnormal: far below half's range */
    int eh = ex - 1023 + 15;
    if (eh >= 31) return (uint16_t)(sign | 0x7C00u);   /* |s| >= 2^16: overflow */
    uint64_t q, rem, half;
    if (eh <= 0) {                              /* half subnormal: units of 2^-24 */
        int shift = 1051 - ex;                  /* m * 2^(ex - 1075) / 2^-24 */
        if (shift >= 54) return sign;           /* below a quarter of the smallest subnormal */
        uint64_t m = man | (1ull << 52);
        q = m >> shift;
        rem = m & ((1ull << shift) - 1);
        half = 1ull << (shift - 1);
    } else {
        q = ((uint64_t)eh << 10) | (man >> 42);
        rem = man & ((1ull << 42) - 1);
        half = 1ull << 41;
    }
    int up;
    if (rem != half) up = rem > half;
    else if (e != 0.0) up = (e > 0.0) == (s > 0.0);   /* e moves the magnitude off the tie */
    else up = (int)(q & 1u);
    if (up) q++;                                /* a carry into the exponent is the correct result */
    return (uint16_t)(sign | (uint16_t)q);
}

/* __hfma(a, b, c): a * b + c rounded once to binary16.  The product of two
 * 11-bit significands is exact in binary64, the sum is split into s + e by
 * TwoSum (Knuth), and s + e is rounded to binary16 in one step. */
uint16_t orc_hfma(uint16_t a, uint16_t b, uint16_t c)
{
    const double fa = orc_f16_to_f32(a), fb = orc_f16_to_f32(b), fc = orc_f16_to_f32(c);
    const double p = fa * fb;
    const double sm = p + fc;
    if (sm != sm || sm == INFINITY || sm == -INFINITY) return orc_f64_to_f16_rn(sm, 0.0);
    const double bv = sm - p;
    const double err = (p - (sm - bv)) + (fc - bv);
    return orc_f64_to_f16_rn(sm, err);
}

/* (int8_t) of a double as the x86-64 host compiler emits it: truncate to
 * int32 (0x80000000 when NaN or out of range), keep the low byte. */
static int8_t trunc_i8(double v)
{
    int32_t w;
    if (v != v || v >= 2147483648.0 || v < -2147483648.0) w = (int32_t)0x80000000u;
    else w = (int32_t)v;
    return (int8_t)(uint8_t)(w & 0xFF);
}

/* Encoder (main-cg-mixed.cu:2333-2350): half = RN(float value) (the float copy
 * is itself RN(double)); int8 = C truncation of the double.  The reference's
 * out-of-range int8 conversion is undefined in C; this restates what the x86-64
 * host compiler emits (truncate to int32, keep the low byte). */
void orc_encode_ref(int n, const double *val, const float *val_low,
                    uint16_t *val_f16, int8_t *val_i8)
{
    for (int i = 0; i < n; i++) {
        val_f16[i] = orc_f32_to_f16_rn(val_low[i]);
        val_i8[i] = trunc_i8(val[i]);
    }
}

/* Scaled INT8 per tile (a design change from the reference's unscaled cast):
 * s_t = max|a| / 127 (float), q = rint(a / s_t) clamped to [-127, 127]. */
void orc_encode_i8_scaled(const orc_tiles *T, int8_t *q, float *scale)
{
    for (int t = 0; t < T->tilenum; t++) {
        int o = T->csr_offset[t], e = T->csr_offset[t + 1];
        double mx = 0.0;
        for (int k = o; k < e; k++) { double a = fabs(T->val[k]); if (a > mx) mx = a; }
        float s = (float)(mx / 127.0);
        scale[t] = s;
        for (int k = o; k < e; k++) {
            if (s == 0.0f) { q[k] = 0; continue; }
            double r = rint(T->val[k] / (double)s);
            if (r > 127.0) r = 127.0;
            if (r < -127.0) r = -127.0;
            q[k] = (int8_t)r;
        }
    }
}

/* Label of one element from |p_new - p_old| (main-cg-mixed.cu:1334-1351). */
int orc_classify_ref(double dp)
{
    if (dp <= 1e-7 && dp > 1e-8) return 2;
    if (dp <= 1e-6 && dp > 1e-7) return 3;
    if (dp <= 1e-5 && dp > 1e-6) return 4;
    if (dp > 1e-5) return 1;
    return 0;
}

/* Segment label (main-cg-mixed.cu:1352-1369): the vis code written per 16-element
 * segment.  The reference keeps whichever lane wrote last; the deterministic
 * restatement keeps the most conservative written class (FP64 > FP32 > FP16 >
 * INT8), which is always one of the reference's possible outcomes.  No write in
 * the segment -> bypass (d_vis = 1).  Output codes: 0 FP64, 4 FP32, 3 FP16,
 * 2 INT8, 1 bypass. */
void orc_segment_labels_ref(int nseg, const double *p_old, const double *p_new, int *vis)
{
    for (int s = 0; s < nseg; s++) {
        int rank = 0;   /* 0 none, 1 int8, 2 fp16, 3 fp32, 4 fp64 */
        for (int i = 0; i < BS; i++) {
            int c = orc_classify_ref(fabs(p_new[s * BS + i] - p_old[s * BS + i]));
            int r = (c == 1) ? 4 : (c == 4) ? 3 : (c == 3) ? 2 : (c == 2) ? 1 : 0;
            if (r > rank) rank = r;
        }
        static const int code[5] = {1, 2, 3, 4, 0};
        vis[s] = code[rank];
    }
}

/* FP64 tile SpMV restating the reference's host verification loop
 * (main-cg-mixed.cu:2966-2994), including its use of the uint8 end offsets. */
void orc_spmv_tile(const orc_tiles *T, const orc_rowlists *L, int rowA,
                   const double *x, double *y, int nthreads)
{
    (void)rowA;
#ifdef _OPENMP
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(static)
#endif
    for (int R = 0; R < T->tilem; R++) {
        double acc[BS];
        for (int ri = 0; ri < BS; ri++) acc[ri] = 0.0;
        for (int t = T->tile_ptr[R]; t < T->tile_ptr[R + 1]; t++) {
            const double *xo = x + (size_t)T->tile_columnidx[t] * BS;
            int off = T->csr_offset[t];
            for (int q = L->nonzero_row_new[t]; q < L->nonzero_row_new[t + 1]; q++) {
                int ro = L->blockrowid_new[q + 1];
                double s = 0.0;
                for (int k = L->blockcsr_ptr_new[q]; k < L->blockcsr_ptr_new[q + 1]; k++)
                    s += xo[T->col[off + k]] * T->val[off + k];
                acc[ro] += s;
            }
        }
        int rl = (R == T->tilem - 1) ? rowA - R * BS : BS;
        for (int ri = 0; ri < rl; ri++) y[(size_t)R * BS + ri] = acc[ri];
    }
}

/* Correct FP64 tile SpMV (int row bounds, no uint8 wrap) used by the FP64
 * oracle solvers: for each row, per-tile partial sums in tile order. */
static void spmv_tile_exact(const orc_tiles *T, int rowA, const double *x, double *y, int nthreads)
{
#ifdef _OPENMP
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(static)
#endif
    for (int R = 0; R < T->tilem; R++) {
        int rl = (R == T->tilem - 1) ? rowA - R * BS : BS;
        double acc[BS];
        for (int ri = 0; ri < BS; ri++) acc[ri] = 0.0;
        for (int t = T->tile_ptr[R]; t < T->tile_ptr[R + 1]; t++) {
            const double *xo = x + (size_t)T->tile_columnidx[t] * BS;
            int off = T->csr_offset[t], nz = T->csr_offset[t + 1] - off;
            const unsigned char *pt = T->ptr + T->csrptr_offset[t];
            for (int ri = 0; ri < rl; ri++) {
                int st = pt[ri], sp = (ri == rl - 1) ? nz : pt[ri + 1];
                double s = 0.0;
                for (int k = st; k < sp; k++) s += xo[T->col[off + k]] * T->val[off + k];
                acc[ri] += s;
            }
        }
        for (int ri = 0; ri < rl; ri++) y[(size_t)R * BS + ri] = acc[ri];
    }
}

/* The stored value of entry e of tile t in precision prec, widened to FP64. */
static double stored_value(const orc_tiles *T, int t, int e, int prec, const uint16_t *v16, const int8_t *q8,
                           const float *scale)
{
    switch (prec) {
    case 0: return T->val[e];
    case 1: return (double)T->val_low[e];
    case 2: return (double)orc_f16_to_f32(v16[e]);
    default: return (double)((float)q8[e] * scale[t]);
    }
}

/* The product of the encoded values (the values the reference's tile SpMV,
 * main-cg-mixed.cu:1130-1214, multiplies in each precision; INT8 with the
 * per-tile scale of this build), accumulated in FP64 in the GPU slice walk's
 * order: per row, tile by tile in slices of 15, payload order within a tile. */
void orc_spmv_slices(const orc_tiles *T, int rowA, const double *x, double *y, int prec,
                     const uint16_t *v16, const int8_t *q8, const float *scale)
{
    for (int R = 0; R < T->tilem; R++) {
        const int rl = (R == T->tilem - 1) ? rowA - R * BS : BS;
        const int t0 = T->tile_ptr[R], t1 = T->tile_ptr[R + 1];
        for (int ri = 0; ri < rl; ri++) {
            double acc = 0.0;
            for (int ts = t0; ts < t1; ts += 15) {
                const int te = (ts + 15 < t1) ? ts + 15 : t1;
                double sacc = 0.0;
                for (int t = ts; t < te; t++) {
                    const double *xo = x + (size_t)T->tile_columnidx[t] * BS;
                    const int off = T->csr_offset[t], nz = T->csr_offset[t + 1] - off;
                    const unsigned char *pt = T->ptr + T->csrptr_offset[t];
                    const int st = pt[ri], sp = (ri == rl - 1) ? nz : pt[ri + 1];
                    for (int k = st; k < sp; k++)
                        sacc = fma(stored_value(T, t, off + k, prec, v16, q8, scale), xo[T->col[off + k]], sacc);
                }
                acc += sacc;
            }
            y[(size_t)R * BS + ri] = acc;
        }
    }
}

/* Tile products of the reference's mixed SpMV (main-cg-mixed.cu:1130-1214):
 * per (tile, row) two partial sums, entries at even / odd positions of the
 * row (the reference's lane pair, virtual_lane_id), in the precision of the
 * column segment's label -- FP64 fma on p, FP32 fmaf on (float)p, FP16 __hfma
 * on half(p), INT8 int8 sums (wrapping) of (int8_t)p times the truncated
 * values, bypass skipped -- each partial widened and added to the row's FP64
 * sum, even then odd, tile by tile.  The reference adds them with atomics in
 * no fixed order; this is the fixed order of the GPU parity mode (per slice of
 * 15 tiles, slice sums added in turn). */
static void spmv_parity(const orc_tiles *T, int rowA, const double *p, const float *p32, const uint16_t *p16,
                        const int8_t *p8, const int *lab, const uint16_t *v16, const int8_t *i8ref, double *y)
{
    for (int R = 0; R < T->tilem; R++) {
        const int rl = (R == T->tilem - 1) ? rowA - R * BS : BS;
        const int t0 = T->tile_ptr[R], t1 = T->tile_ptr[R + 1];
        for (int ri = 0; ri < rl; ri++) {
            double acc = 0.0;
            for (int ts = t0; ts < t1; ts += 15) {
                const int te = (ts + 15 < t1) ? ts + 15 : t1;
                double sacc = 0.0;
                for (int t = ts; t < te; t++) {
                    const int j = T->tile_columnidx[t];
                    const int code = lab[j];
                    const int off = T->csr_offset[t], nz = T->csr_offset[t + 1] - off;
                    const unsigned char *pt = T->ptr + T->csrptr_offset[t];
                    const int st = pt[ri], sp = (ri == rl - 1) ? nz : pt[ri + 1];
                    if (code == 1 || st >= sp) continue;
                    double a64[2] = {0.0, 0.0};
                    float a32[2] = {0.0f, 0.0f};
                    uint16_t a16[2] = {0, 0};
                    int8_t a8[2] = {0, 0};
                    for (int k = st; k < sp; k++) {
                        const int e = off + k, q = (k - st) & 1;
                        const size_t col = (size_t)j * BS + T->col[e];
                        if (code == 0) a64[q] = fma(p[col], T->val[e], a64[q]);
                        else if (code == 4) a32[q] = fmaf(p32[col], T->val_low[e], a32[q]);
                        else if (code == 3) a16[q] = orc_hfma(p16[col], v16[e], a16[q]);
                        else a8[q] = (int8_t)((int)a8[q] + (int)p8[col] * (int)i8ref[e]);
                    }
                    for (int q = 0; q < 2; q++) {
                        if (code == 0) sacc += a64[q];
                        else if (code == 4) sacc += (double)a32[q];
                        else if (code == 3) sacc += (double)orc_f16_to_f32(a16[q]);
                        else sacc += (double)a8[q];
                    }
                }
                acc += sacc;
            }
            y[(size_t)R * BS + ri] = acc;
        }
    }
}

static double dot_seq(int n, const double *a, const double *b)
{
    double t = 0.0;
    for (int i = 0; i < n; i++) t += a[i] * b[i];
    return t;
}

/* Parity-mode CG (main-cg-mixed.cu:1115-1385), the reference's three phases
 * per iteration: q = A p with the label-selected tile arithmetic, alpha =
 * r.r / p.q, r -= alpha q, beta = r'.r' / r.r, x += alpha p, p = r + beta p;
 * then p's shadows (float)p, half(p) (__double2half, one rounding) and
 * (int8_t)p (the int8 conversion of main-cg-mixed.cu:435) and the labels of
 * the next SpMV from |p_new - p_old| per 16-element segment (thresholds of
 * main-cg-mixed.cu:1334-1351).  The reference keeps the class of whichever
 * lane wrote last; here the most conservative class wins (one of the
 * reference's possible outcomes) and agree[s] says whether every lane of the
 * segment had the same class (the reference's label is then determined).
 * x0 = 0, labels start all FP64 (cudaMemset(d_vis, 0), main-cg-mixed.cu:2828).
 * Dot products are sequential sums.  The axpys use fma as nvcc contracts
 * them. */
int orc_cg_parity(const orc_tiles *T, int n, const double *b, const uint16_t *v16, const int8_t *i8ref,
                  double *x, int iters, int *labels, int *agree, orc_report *rep)
{
    const size_t N = vec_len(T, n);
    const int nseg = (int)(N / BS);
    double *r = (double *)calloc(N, sizeof(double));
    double *p = (double *)calloc(N, sizeof(double));
    double *q = (double *)calloc(N, sizeof(double));
    double *xx = (double *)calloc(N, sizeof(double));
    double *pold = (double *)calloc(N, sizeof(double));
    float *p32 = (float *)calloc(N, sizeof(float));
    uint16_t *p16 = (uint16_t *)calloc(N, sizeof(uint16_t));
    int8_t *p8 = (int8_t *)calloc(N, sizeof(int8_t));
    int *lab = (int *)calloc((size_t)nseg, sizeof(int));
    int *agr = (int *)calloc((size_t)nseg, sizeof(int));
    for (int i = 0; i < n; i++) {
        r[i] = b[i];
        p[i] = b[i];
        p32[i] = (float)b[i];
        p16[i] = orc_f64_to_f16_rn(b[i], 0.0);
        p8[i] = trunc_i8(b[i]);
    }
    for (int s = 0; s < nseg; s++) agr[s] = 1;
    double rr = dot_seq(n, r, r);
    const double bb = rr;
    for (int k = 0; k < iters; k++) {
        spmv_parity(T, n, p, p32, p16, p8, lab, v16, i8ref, q);
        const double alpha = rr / dot_seq(n, p, q);
        for (int i = 0; i < n; i++) r[i] = fma(-alpha, q[i], r[i]);
        const double rr_new = dot_seq(n, r, r);
        const double beta = rr_new / rr;
        rr = rr_new;
        memcpy(pold, p, N * sizeof(double));
        for (int i = 0; i < n; i++) {
            xx[i] = fma(alpha, pold[i], xx[i]);
            p[i] = fma(beta, pold[i], r[i]);
            p32[i] = (float)p[i];
            p16[i] = orc_f64_to_f16_rn(p[i], 0.0);
            p8[i] = trunc_i8(p[i]);
        }
        for (int s = 0; s < nseg; s++) {
            int rank = 0, c0 = -1, same = 1;
            for (int i = s * BS; i < s * BS + BS && i < n; i++) {
                const int c = orc_classify_ref(fabs(p[i] - pold[i]));
                const int rk = (c == 1) ? 4 : (c == 4) ? 3 : (c == 3) ? 2 : (c == 2) ? 1 : 0;
                if (rk > rank) rank = rk;
                if (c0 < 0) c0 = c;
                else if (c != c0) same = 0;
            }
            static const int code[5] = {1, 2, 3, 4, 0};
            lab[s] = code[rank];
            agr[s] = same;
        }
    }
    spmv_tile_exact(T, n, xx, q, 1);
    double rt = 0.0;
    for (int i = 0; i < n; i++) { const double d = b[i] - q[i]; rt += d * d; }
    memcpy(x, xx, (size_t)n * sizeof(double));
    if (labels) memcpy(labels, lab, (size_t)T->tilen * sizeof(int));
    if (agree) memcpy(agree, agr, (size_t)T->tilen * sizeof(int));
    if (rep) {
        rep->iterations = iters;
        rep->converged = 0;
        rep->relres_rec = bb > 0 ? sqrt(rr / bb) : 0.0;
        rep->relres_true = bb > 0 ? sqrt(rt / bb) : 0.0;
        rep->replacements = 0;
    }
    free(r); free(p); free(q); free(xx); free(pold); free(p32); free(p16); free(p8); free(lab); free(agr);
    return 0;
}

void orc_csr_spmv(int n, const int *rowptr, const int *colidx, const double *val,
                  const double *x, double *y, int nthreads)
{
#ifdef _OPENMP
    if (nthreads < 1) nthreads = 1;
#pragma omp parallel for num_threads(nthreads) schedule(static)
#endif
    for (int i = 0; i < n; i++) {
        double s = 0.0;
        for (int j = rowptr[i]; j < rowptr[i + 1]; j++) s += val[j] * x[colidx[j]];
        y[i] = s;
    }
}

/* itsol_dot (Mille-feuille-bicg.h:21-29), optionally threaded (fixed chunking). */
static double dot(int n, const double *a, const double *b, int nthreads)
{
    double t = 0.0;
#ifdef _OPENMP
    if (nthreads > 1) {
#pragma omp parallel for num_threads(nthreads) reduction(+:t) schedule(static)
        for (int i = 0; i < n; i++) t += a[i] * b[i];
        return t;
    }
#endif
    (void)nthreads;
    for (int i = 0; i < n; i++) t += a[i] * b[i];
    return t;
}

/* x vectors are sized to cover every column tile (tilen*16) so that column
 * tiles past the truncated row count read zeros, as in the reference's padded
 * device buffers (main-cg-mixed.cu:2813-2824). */
static size_t vec_len(const orc_tiles *T, int n)
{
    size_t a = (size_t)T->tilen * BS, b = (size_t)T->tilem * BS;
    size_t m = a > b ? a : b;
    return m > (size_t)n ? m : (size_t)n;
}

/* FP64 CG: the alpha/beta schedule of Mille-feuille-cg.h:1237-1370 /
 * main-cg.cu:258-292 (alpha = r.r / p.Ap; x += alpha p; r -= alpha Ap;
 * beta = r'.r' / r.r; p = r + beta p), x0 = 0, plus a convergence stop:
 * when the recursive ||r|| <= tol ||b|| the true residual b - A x is formed
 * in FP64; the solve ends if it also passes, otherwise r is replaced by it. */
int orc_cg_fp64(const orc_tiles *T, const orc_rowlists *L, int n,
                const double *b, double *x, double tol, int max_iter,
                int fixed_iters, int nthreads, orc_report *rep)
{
    (void)L;
    size_t N = vec_len(T, n);
    double *r = (double *)calloc(N, sizeof(double));
    double *p = (double *)calloc(N, sizeof(double));
    double *q = (double *)calloc(N, sizeof(double));
    double *xx = (double *)calloc(N, sizeof(double));
    for (int i = 0; i < n; i++) { r[i] = b[i]; p[i] = b[i]; }
    double bnorm = sqrt(dot(n, b, b, nthreads));
    double thr = tol * bnorm;
    double rr = dot(n, r, r, nthreads);
    int k = 0, conv = 0, repl = 0;
    for (;;) {
        if (!fixed_iters && sqrt(rr) <= thr) {
            spmv_tile_exact(T, n, xx, q, nthreads);
            for (int i = 0; i < n; i++) q[i] = b[i] - q[i];
            double rt = dot(n, q, q, nthreads);
            if (sqrt(rt) <= thr) { conv = 1; break; }
            memcpy(r, q, (size_t)n * sizeof(double));
            rr = rt;
            repl++;
        }
        if (k >= max_iter) break;
        spmv_tile_exact(T, n, p, q, nthreads);
        double pq = dot(n, p, q, nthreads);
        double alpha = rr / pq;
        for (int i = 0; i < n; i++) { xx[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
        double rr_new = dot(n, r, r, nthreads);
        double beta = rr_new / rr;
        rr = rr_new;
        for (int i = 0; i < n; i++) p[i] = r[i] + beta * p[i];
        k++;
    }
    spmv_tile_exact(T, n, xx, q, nthreads);
    double rt = 0.0;
    for (int i = 0; i < n; i++) { double d = b[i] - q[i]; rt += d * d; }
    memcpy(x, xx, (size_t)n * sizeof(double));
    if (rep) {
        rep->iterations = k;
        rep->converged = conv;
        rep->relres_rec = bnorm > 0 ? sqrt(rr) / bnorm : 0.0;
        rep->relres_true = bnorm > 0 ? sqrt(rt) / bnorm : 0.0;
        rep->replacements = repl;
    }
    free(r); free(p); free(q); free(xx);
    return conv ? 0 : 1;
}

/* FP64 BiCGSTAB with the reference's formulas (main-bicg.cu:1619-1656 and the
 * kernels of Mille-feuille-bicg.h:47-86): alpha = r1 / (rh.v), s = r - alpha v,
 * omega = (t.s)/(t.t), x += alpha p + omega s, r = s - omega t,
 * beta = (r1' alpha) / (r1 omega), p = r + beta (p - omega v); x0 = 0, rh = r0.
 * Stop: recursive ||r|| (or ||s||) <= tol ||b||, confirmed by the true residual. */
int orc_bicgstab_fp64(const orc_tiles *T, const orc_rowlists *L, int n,
                      const double *b, double *x, double tol, int max_iter,
                      int fixed_iters, int nthreads, orc_report *rep)
{
    (void)L;
    size_t N = vec_len(T, n);
    double *r = (double *)calloc(N, sizeof(double));
    double *rh = (double *)calloc(N, sizeof(double));
    double *p = (double *)calloc(N, sizeof(double));
    double *v = (double *)calloc(N, sizeof(double));
    double *s = (double *)calloc(N, sizeof(double));
    double *t = (double *)calloc(N, sizeof(double));
    double *xx = (double *)calloc(N, sizeof(double));
    for (int i = 0; i < n; i++) { r[i] = b[i]; rh[i] = b[i]; p[i] = b[i]; }
    double bnorm = sqrt(dot(n, b, b, nthreads));
    double thr = tol * bnorm;
    double r1 = dot(n, r, rh, nthreads);
    double res = sqrt(dot(n, r, r, nthreads));
    int k = 0, conv = 0, repl = 0;
    for (;;) {
        if (!fixed_iters && res <= thr) {
            spmv_tile_exact(T, n, xx, t, nthreads);
            for (int i = 0; i < n; i++) t[i] = b[i] - t[i];
            double rt = sqrt(dot(n, t, t, nthreads));
            if (rt <= thr) { conv = 1; break; }
            memcpy(r, t, (size_t)n * sizeof(double));
            res = rt;
            r1 = dot(n, r, rh, nthreads);
            repl++;
        }
        if (k >= max_iter) break;
        double r0 = r1;
        spmv_tile_exact(T, n, p, v, nthreads);
        double alpha = r0 / dot(n, rh, v, nthreads);
        for (int i = 0; i < n; i++) s[i] = r[i] - alpha * v[i];
        spmv_tile_exact(T, n, s, t, nthreads);
        double ts = dot(n, t, s, nthreads), tt = dot(n, t, t, nthreads);
        double omega = (tt != 0.0) ? ts / tt : 0.0;
        for (int i = 0; i < n; i++) {
            xx[i] = xx[i] + alpha * p[i] + omega * s[i];
            r[i] = s[i] - omega * t[i];
        }
        res = sqrt(dot(n, r, r, nthreads));
        r1 = dot(n, r, rh, nthreads);
        double beta = (r1 * alpha) / (r0 * omega);
        for (int i = 0; i < n; i++) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        k++;
    }
    spmv_tile_exact(T, n, xx, t, nthreads);
    double rt = 0.0;
    for (int i = 0; i < n; i++) { double d = b[i] - t[i]; rt += d * d; }
    memcpy(x, xx, (size_t)n * sizeof(double));
    if (rep) {
        rep->iterations = k;
        rep->converged = conv;
        rep->relres_rec = bnorm > 0 ? res / bnorm : 0.0;
        rep->relres_true = bnorm > 0 ? sqrt(rt) / bnorm : 0.0;
        rep->replacements = repl;
    }
    free(r); free(rh); free(p); free(v); free(s); free(t); free(xx);
    return conv ? 0 : 1;
}

/* ---- Matrix Market reader: mmio_info + mmio_data (mmio_highlevel.h:7-323) ---- */

static char *next_tok(char **pp)
{
    char *p = *pp;
    while (*p && isspace((unsigned char)*p)) p++;
    if (!*p) { *pp = p; return NULL; }
    char *s = p;
    while (*p && !isspace((unsigned char)*p)) p++;
    *pp = p;
    return s;
}

int orc_read_mtx(const char *path, int *m, int *n, int *nnz, int **rowptr,
                 int **colidx, double **val, int *is_sym)
{
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *buf = (char *)malloc((size_t)sz + 1);
    if (fread(buf, 1, (size_t)sz, f) != (size_t)sz) { fclose(f); free(buf); return -1; }
    buf[sz] = 0;
    fclose(f);
    /* banner (mmio.h mm_read_banner): 5 tokens, fields lower-cased */
    char *line_end = strchr(buf, '\n');
    if (!line_end) { free(buf); return -2; }
    *line_end = 0;
    char b0[64] = {0}, b1[64] = {0}, b2[64] = {0}, b3[64] = {0}, b4[64] = {0};
    if (sscanf(buf, "%63s %63s %63s %63s %63s", b0, b1, b2, b3, b4) != 5) { free(buf); return -2; }
    for (char *q = b2; *q; q++) *q = (char)tolower((unsigned char)*q);
    for (char *q = b3; *q; q++) *q = (char)tolower((unsigned char)*q);
    for (char *q = b4; *q; q++) *q = (char)tolower((unsigned char)*q);
    if (strncmp(b0, "%%MatrixMarket", 14) != 0 || strcmp(b2, "coordinate") != 0) { free(buf); return -2; }
    int isPattern = !strcmp(b3, "pattern"), isReal = !strcmp(b3, "real");
    int isComplex = !strcmp(b3, "complex"), isInteger = !strcmp(b3, "integer");
    int sym = !strcmp(b4, "symmetric") || !strcmp(b4, "hermitian");
    char *p = line_end + 1;
    /* skip comment lines (mm_read_mtx_crd_size) */
    while (*p == '%') { char *e = strchr(p, '\n'); if (!e) { free(buf); return -4; } p = e + 1; }
    long long M = strtoll(p, &p, 10), Ncol = strtoll(p, &p, 10), NZ = strtoll(p, &p, 10);
    if (M <= 0 || Ncol <= 0 || NZ < 0) { free(buf); return -4; }
    int *ri = (int *)malloc(((size_t)NZ + 1) * sizeof(int));
    int *ci = (int *)malloc(((size_t)NZ + 1) * sizeof(int));
    double *vv = (double *)malloc(((size_t)NZ + 1) * sizeof(double));
    long long *cnt = (long long *)calloc((size_t)M + 1, sizeof(long long));
    for (long long i = 0; i < NZ; i++) {
        char *t1 = next_tok(&p), *t2 = next_tok(&p);
        if (!t1 || !t2) { free(buf); free(ri); free(ci); free(vv); free(cnt); return -5; }
        int a = (int)strtol(t1, NULL, 10) - 1, c = (int)strtol(t2, NULL, 10) - 1;
        double fv = 1.0;
        if (isReal) fv = strtod(next_tok(&p), NULL);
        else if (isComplex) { fv = strtod(next_tok(&p), NULL); (void)next_tok(&p); }
        else if (isInteger) fv = (double)(int)strtol(next_tok(&p), NULL, 10);
        else if (isPattern) fv = 1.0;
        ri[i] = a; ci[i] = c; vv[i] = fv;
        cnt[a]++;
    }
    free(buf);
    if (sym) for (long long i = 0; i < NZ; i++) if (ri[i] != ci[i]) cnt[ci[i]]++;
    /* exclusive scan */
    long long prev = cnt[0];
    cnt[0] = 0;
    for (long long i = 1; i <= M; i++) { long long cur = cnt[i]; cnt[i] = prev + cnt[i - 1]; prev = cur; }
    long long total = cnt[M];
    int *rp = (int *)malloc(((size_t)M + 1) * sizeof(int));
    for (long long i = 0; i <= M; i++) rp[i] = (int)cnt[i];
    int *cc = (int *)malloc(((size_t)total + 1) * sizeof(int));
    double *vo = (double *)malloc(((size_t)total + 1) * sizeof(double));
    long long *fill = (long long *)calloc((size_t)M + 1, sizeof(long long));
    for (long long i = 0; i < NZ; i++) {
        long long o = cnt[ri[i]] + fill[ri[i]]++;
        cc[o] = ci[i]; vo[o] = vv[i];
        if (sym && ri[i] != ci[i]) {
            o = cnt[ci[i]] + fill[ci[i]]++;
            cc[o] = ri[i]; vo[o] = vv[i];
        }
    }
    free(ri); free(ci); free(vv); free(cnt); free(fill);
    *m = (int)M; *n = (int)Ncol; *nnz = (int)total;
    *rowptr = rp; *colidx = cc; *val = vo; *is_sym = sym;
    return 0;
}
