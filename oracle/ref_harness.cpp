/*
 * ref_harness.cpp -- exposes the reference's own host code (compiled from the
 * reference sources where they lie, never copied) behind a small C ABI so that
 * tests can pin the oracle restatement against it.
 *
 * TEST INFRASTRUCTURE ONLY.  Built by oracle/Makefile into
 * oracle/_ref/libmf_refhost.so when the reference tree is present.
 *
 * Wrapped reference functions:
 *   Tile_create         (csr2block.h:267-422)
 *   blockspmv_cpu       (blockspmv_cpu.h:2-112)  -- offsets only (x = 0)
 *   read_Dmatrix_32     (biio2.0/src/biio.h:153-194)
 */
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "csr2block.h"
#include "blockspmv_cpu.h"
#include "./biio2.0/src/biio.h"

extern "C" {

struct ref_tiles {
    Tile_matrix m;
    int rowA;
    int *ptroffset1, *ptroffset2;
    int rowblkblock;
    unsigned int *rb_idx;
    int *rb_start, *rb_stop;
};

void *ref_tile_create(int rowA, int colA, int nnz, const int *rowptr, const int *colidx,
                      const double *val, const float *val_low)
{
    ref_tiles *h = (ref_tiles *)calloc(1, sizeof(ref_tiles));
    h->rowA = rowA;
    Tile_create(&h->m, rowA, colA, nnz, (int *)rowptr, (int *)colidx, (double *)val, (float *)val_low);
    int tn = h->m.tilenum;
    h->ptroffset1 = (int *)calloc(tn + 1, sizeof(int));
    h->ptroffset2 = (int *)calloc(tn + 1, sizeof(int));
    int ylen = h->m.tilem * BLOCK_SIZE + BLOCK_SIZE;
    int xlen = h->m.tilen * BLOCK_SIZE + BLOCK_SIZE;
    double *x = (double *)calloc(xlen, sizeof(double));
    double *y = (double *)calloc(ylen, sizeof(double));
    double *yg = (double *)calloc(ylen, sizeof(double));
    blockspmv_cpu(&h->m, h->ptroffset1, h->ptroffset2, &h->rowblkblock, &h->rb_idx,
                  &h->rb_start, &h->rb_stop, rowA, colA, nnz, (int *)rowptr, (int *)colidx,
                  (double *)val, x, y, yg);
    free(x); free(y); free(yg);
    return h;
}

/* dims: tilem, tilen, tilenum, csrsize, csrptrlen, rowblkblock */
void ref_tile_dims(void *hp, int *dims)
{
    ref_tiles *h = (ref_tiles *)hp;
    dims[0] = h->m.tilem; dims[1] = h->m.tilen; dims[2] = h->m.tilenum;
    dims[3] = h->m.csrsize; dims[4] = h->m.csrptrlen; dims[5] = h->rowblkblock;
}

/* Copy one array out by name. */
int ref_tile_get(void *hp, const char *name, void *dst)
{
    ref_tiles *h = (ref_tiles *)hp;
    Tile_matrix *m = &h->m;
    int tm = m->tilem, tn = m->tilenum;
    if (!strcmp(name, "tile_ptr")) memcpy(dst, m->tile_ptr, (tm + 1) * sizeof(int));
    else if (!strcmp(name, "tile_columnidx")) memcpy(dst, m->tile_columnidx, tn * sizeof(int));
    else if (!strcmp(name, "tile_nnz")) memcpy(dst, m->tile_nnz, (tn + 1) * sizeof(int));
    else if (!strcmp(name, "blknnz")) memcpy(dst, m->blknnz, (tn + 1) * sizeof(int));
    else if (!strcmp(name, "csr_offset")) memcpy(dst, m->csr_offset, (tn + 1) * sizeof(int));
    else if (!strcmp(name, "csrptr_offset")) memcpy(dst, m->csrptr_offset, (tn + 1) * sizeof(int));
    else if (!strcmp(name, "val")) memcpy(dst, m->Blockcsr_Val, m->csrsize * sizeof(double));
    else if (!strcmp(name, "val_low")) memcpy(dst, m->Blockcsr_Val_Low, m->csrsize * sizeof(float));
    else if (!strcmp(name, "col")) memcpy(dst, m->Tile_csr_Col, m->csrsize);
    else if (!strcmp(name, "ptr")) memcpy(dst, m->Blockcsr_Ptr, m->csrptrlen);
    else if (!strcmp(name, "ptroffset1")) memcpy(dst, h->ptroffset1, tn * sizeof(int));
    else if (!strcmp(name, "ptroffset2")) memcpy(dst, h->ptroffset2, tn * sizeof(int));
    else if (!strcmp(name, "blkcoostylerowidx")) memcpy(dst, h->rb_idx, h->rowblkblock * sizeof(unsigned int));
    else if (!strcmp(name, "colstart")) memcpy(dst, h->rb_start, h->rowblkblock * sizeof(int));
    else if (!strcmp(name, "colstop")) memcpy(dst, h->rb_stop, h->rowblkblock * sizeof(int));
    else return -1;
    return 0;
}

void ref_tile_free(void *hp)
{
    ref_tiles *h = (ref_tiles *)hp;
    free(h->ptroffset1); free(h->ptroffset2);
    free(h->rb_idx); free(h->rb_start); free(h->rb_stop);
    Tile_matrix *m = &h->m;
    free(m->tile_ptr); free(m->tile_columnidx); free(m->tile_nnz); free(m->Format);
    free(m->blknnz); free(m->blknnznnz); free(m->tilewidth); free(m->csr_offset);
    free(m->csrptr_offset); free(m->Blockcsr_Val); free(m->Blockcsr_Val_Low);
    free(m->Blockcsr_Ptr); free(m->csr_compressedIdx); free(m->Tile_csr_Col);
    free(h);
}

/* read_Dmatrix_32 on a .mtx / .cbd path. */
int ref_read_matrix(const char *path, int *m, int *n, int *nnz, int **rowptr, int **colidx,
                    double **val, int *is_sym)
{
    *is_sym = 0;
    read_Dmatrix_32(m, n, nnz, rowptr, colidx, val, is_sym, (char *)path);
    return 0;
}

void ref_free(void *p) { free(p); }

}  /* extern "C" */
