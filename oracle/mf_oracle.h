/*
 * mf_oracle.h -- CPU restatement of Mille-feuille's tile path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the test oracle: tests/, the
 * smoke() entry and bench.py's cpu_baseline / reference arm may call it.
 * The product (libmillefeuille.so) never links or calls it.
 *
 * Every function cites the reference file:line (paths inside the
 * zhaijiaqi/Mille-feuille project) whose behaviour it restates.  The
 * restatement is pinned against the reference's own Tile_create /
 * blockspmv_cpu / mmio_data compiled from source into oracle/_ref
 * (see oracle/Makefile) and against the committed fixtures in
 * tests/golden/.
 */
#ifndef MF_ORACLE_H
#define MF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* The fields of Tile_matrix (format.h:14-86) that the CSR-in-tile path
 * actually populates (csr2block.h:267-422 forces Format=0). */
typedef struct {
    int tilem, tilen, tilenum, csrsize, csrptrlen;
    int *tile_ptr;          /* [tilem+1]   */
    int *tile_columnidx;    /* [tilenum]   */
    int *tile_nnz;          /* [tilenum+1] exclusive scan */
    int *blknnz;            /* [tilenum+1] exclusive scan */
    int *csr_offset;        /* [tilenum+1] exclusive scan */
    int *csrptr_offset;     /* [tilenum+1] exclusive scan */
    double *val;            /* Blockcsr_Val     [csrsize] */
    float *val_low;         /* Blockcsr_Val_Low [csrsize] */
    unsigned char *col;     /* Tile_csr_Col     [csrsize] */
    unsigned char *ptr;     /* Blockcsr_Ptr     [csrptrlen] */
} orc_tiles;

/* Nonempty-row lists built inside cg_solve_inc (main-cg-mixed.cu:2447-2514). */
typedef struct {
    int cnt;                        /* nonzero_row_new[tilenum] */
    int *nonzero_row_new;           /* [tilenum+1] */
    unsigned char *blockrowid_new;  /* [cnt+1] */
    unsigned char *blockcsr_ptr_new;/* [cnt+1] */
    int *tile_rowidx;               /* [tilenum] */
    int *block_signal;              /* [tilem+4] */
} orc_rowlists;

/* blockspmv_cpu offsets and row-block split (blockspmv_cpu.h:2-83). */
typedef struct {
    int *ptroffset1;        /* [tilenum] */
    int *ptroffset2;        /* [tilenum] */
    int rowblkblock;
    unsigned int *blkcoostylerowidx;  /* [rowblkblock] */
    int *colstart;          /* [rowblkblock] */
    int *colstop;           /* [rowblkblock] */
} orc_offsets;

int  orc_tile_create(int rowA, int colA, const int *rowptr, const int *colidx,
                     const double *val, const float *val_low, orc_tiles *T);
void orc_tiles_free(orc_tiles *T);
int  orc_offsets_build(const orc_tiles *T, int rowA, orc_offsets *O);
void orc_offsets_free(orc_offsets *O);
int  orc_rowlists_build(const orc_tiles *T, int rowA, orc_rowlists *L);
void orc_rowlists_free(orc_rowlists *L);

/* Precision encoder (main-cg-mixed.cu:2333-2350). */
void orc_encode_ref(int n, const double *val, const float *val_low,
                    uint16_t *val_f16, int8_t *val_i8);
uint16_t orc_f32_to_f16_rn(float f);
float    orc_f16_to_f32(uint16_t h);
/* Per-tile scaled INT8 (design change): s = max|a|/127, q = rint(a/s). */
void orc_encode_i8_scaled(const orc_tiles *T, int8_t *q, float *scale);

/* Reference label classification of one element (main-cg-mixed.cu:1334-1369).
 * Returns the vis code the reference would write: 1 = FP64, 4 = FP32,
 * 3 = FP16, 2 = INT8, 0 = no write (|dp| <= 1e-8 or NaN -> bypass). */
int  orc_classify_ref(double dp);
/* Deterministic segment label: the most conservative class among the 16
 * elements of a segment, mapped to d_vis codes 0 (FP64), 4, 3, 2, 1 (bypass). */
void orc_segment_labels_ref(int nseg, const double *p_old, const double *p_new,
                            int *vis);

/* FP64 tile SpMV, restating the reference's host verification loop
 * (main-cg-mixed.cu:2966-2994): y[16R+ro] += sum over tiles of row ro. */
void orc_spmv_tile(const orc_tiles *T, const orc_rowlists *L, int rowA,
                   const double *x, double *y, int nthreads);

/* Solver report. */
typedef struct {
    int iterations;
    int converged;
    double relres_rec;      /* recursive ||r||/||b|| */
    double relres_true;     /* ||b - A x||/||b|| in FP64 */
    int replacements;
} orc_report;

/* FP64 CG with the reference's alpha/beta schedule (main-cg.cu:258-292,
 * Mille-feuille-cg.h:1113-1348), stopping at relres <= tol (recursive, then
 * confirmed with the true residual).  n = rowA (multiple of 16 not needed). */
int orc_cg_fp64(const orc_tiles *T, const orc_rowlists *L, int n,
                const double *b, double *x, double tol, int max_iter,
                int fixed_iters, int nthreads, orc_report *rep);

/* FP64 BiCGSTAB with the reference's formulas (main-bicg.cu:1619-1656). */
int orc_bicgstab_fp64(const orc_tiles *T, const orc_rowlists *L, int n,
                      const double *b, double *x, double tol, int max_iter,
                      int fixed_iters, int nthreads, orc_report *rep);

/* binary64 value s + e (|e| below half an ulp of s, e.g. TwoSum's error
 * term) -> binary16, round to nearest, ties to even, with e deciding a tie of
 * s alone.  e = 0: the conversion __double2half performs. */
uint16_t orc_f64_to_f16_rn(double s, double e);
/* a * b + c rounded once to binary16 (the semantics of CUDA's __hfma). */
uint16_t orc_hfma(uint16_t a, uint16_t b, uint16_t c);

/* y = A x with every tile's values in one stored precision, in the order the
 * GPU slice walk accumulates: per row, the entries tile by tile in payload
 * order, fma-folded into an FP64 sum that starts at 0 for each slice of
 * <= 15 consecutive tiles; the slice sums are added in turn.  prec: 0 FP64
 * values, 1 FP32 (val_low), 2 FP16 (v16 bits, RN of val_low), 3 scaled INT8
 * (q8 times the tile's float scale, product in float).  The stored value is
 * widened to FP64 and multiplied with the FP64 x. */
void orc_spmv_slices(const orc_tiles *T, int rowA, const double *x, double *y, int prec,
                     const uint16_t *v16, const int8_t *q8, const float *scale);

/* Parity-mode CG: the reference's mixed single-kernel CG
 * (main-cg-mixed.cu:1115-1385) on `iters` fixed iterations from x0 = 0, with
 * the labels of the next SpMV in *labels (tilen codes: 0 FP64, 4 FP32, 3 FP16,
 * 2 INT8, 1 bypass) and, per segment, whether every lane's class agreed
 * (agree, nullable).  v16 / i8ref: the reference encoder's FP16 and truncated
 * INT8 values (orc_encode_ref). */
int orc_cg_parity(const orc_tiles *T, int n, const double *b, const uint16_t *v16, const int8_t *i8ref,
                  double *x, int iters, int *labels, int *agree, orc_report *rep);

/* CSR SpMV y = A x over rows [0,n) (Mille-feuille-bicg.h:31-41 `mv`). */
void orc_csr_spmv(int n, const int *rowptr, const int *colidx, const double *val,
                  const double *x, double *y, int nthreads);

/* Matrix Market reader restating mmio_data (mmio_highlevel.h:151-323):
 * file-order placement, symmetric expansion, pattern -> 1.0.  Returns 0 on
 * success.  The rowptr, colidx and val arrays are malloc'd; caller frees with orc_free. */
int  orc_read_mtx(const char *path, int *m, int *n, int *nnz, int **rowptr,
                  int **colidx, double **val, int *is_sym);
void orc_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
