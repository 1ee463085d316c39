// mf_internal.cuh -- shared device/host definitions of libmillefeuille.
//
// Device data layout (all device-resident, built on the GPU from CSR):
//
//  Reference tile layout (bit-exact to Tile_create, csr2block.h:267-422):
//    tile_ptr[tilem+1], tile_columnidx[T], csr_offset[T+1] (== tile_nnz ==
//    blknnz), csrptr_offset[T+1], val[nnz] f64, val_low[nnz] f32, col[nnz] u8,
//    ptr[csrptrlen] u8, plus the nonempty-row lists of main-cg-mixed.cu:2447-2514.
//
//  Solver slices (this library's own format, derived from the tiles):
//    a tile-row's tiles are cut into segments of <= 15 consecutive tiles; a
//    segment is a 16-row slice stored as a padded ELL block of Kp columns
//    (Kp = max row length in the slice rounded up to 8), i.e. Kp / 8 chunks
//    of 16 rows x 8 entries (128 entries) back to back.  Within a chunk, row
//    i's 8 entries are split into 16-byte groups of g = 16 / element size
//    entries (2 FP64, 4 FP32, 8 FP16 / INT8 / index bytes) and group q of the
//    16 rows sits together (mf_slot below), so lane i reads its row with one
//    128-bit load per group and a half-warp's load covers 256 contiguous bytes
//    (128 for the 8-byte rows of INT8 values and index bytes):
//      meta[mf_slot<1>(off, k, i)]      u8  (slot << 4) | local column
//      v64 / v32 / v16 / v8[mf_slot<size>(off, k, i)]  entry k of row i
//    entries of row i appear tile by tile (slot order), within a tile in the
//    reference payload order.  Per tile: int8 scale and capability flags.
#pragma once
#include <cmath>

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "../../include/millefeuille.h"

#define MF_BS 16
#define MF_SEG_TILES 15

// tile capability / lossless-class bits (tile_caps)
#define MF_CAP_FP16_OK 0x1      // |a| within fp16 normal range (no overflow / subnormal loss)
#define MF_CAP_EXACT_I8 0x2     // scaled int8 reproduces every value exactly
#define MF_CAP_EXACT_F16 0x4    // fp16 reproduces every value exactly
#define MF_CAP_EXACT_F32 0x8    // fp32 reproduces every value exactly

// per-entry precision codes used inside the solver
#define MF_P64 0
#define MF_P32 1
#define MF_P16 2
#define MF_P8 3
#define MF_PSKIP 4

struct mf_matrix_s {
    int dev;
    int n_rows, n_cols;        // as given
    long long nnz;             // entries in rows [0, n_rows)
    int tilem, tilen, tilenum;
    int csrsize, csrptrlen, cnt_non_new, rowblkblock;
    int vec_len;               // max(tilem, tilen) * 16: padded vector length
    // input CSR (device copies)
    int *d_rowptr, *d_colidx;
    double *d_val;
    float *d_val_low;
    // reference layout
    int *d_tile_ptr, *d_tile_columnidx, *d_csr_offset, *d_csrptr_offset;
    double *d_tval;
    float *d_tval_low;
    unsigned char *d_tcol, *d_tptr;
    int *d_nonzero_row_new, *d_tile_rowidx, *d_block_signal;
    unsigned char *d_blockrowid_new, *d_blockcsr_ptr_new;
    unsigned int *d_rb_idx;
    int *d_rb_start, *d_rb_stop;
    uint16_t *d_val_f16;       // encoder: RN(float) half bits, reference payload order
    int8_t *d_val_i8_ref;      // encoder: reference (int8_t) truncation
    int8_t *d_val_i8;          // encoder: scaled int8 (reference payload order)
    float *d_i8_scale;         // per tile
    unsigned char *d_tile_caps;// per tile
    // solver slices
    int nseg;
    int *d_seg_ptr;            // [tilem+1]
    int *d_seg_tile0;          // [nseg+1] first tile of each segment (+ end)
    long long *d_seg_off;      // [nseg+1] entry offset
    int4 *d_seg_hdr;           // [nseg+1] {first tile, tile-row, kp | ntiles << 16 | last << 24, offset / 128}
    int *d_seg_tile;           // [nseg*16] tile words: column-tile << 8 | caps (0 past the slice's tiles)
    int *d_seg_kp;             // [nseg]
    uint16_t *d_seg_rowlen;    // [nseg*16]
    long long slice_entries;
    unsigned char *d_meta;
    double *d_v64;
    float *d_v32;
    __half *d_v16;
    int8_t *d_v8;
    int8_t *d_v8ref;           // reference (unscaled, truncated) int8 values, parity mode only
    // tile-row ownership cost prefix for partitioning: [tilem+1]
    long long *d_row_cost;
    double build_ms;
    // cached solver workspace
    void *ws;
    size_t ws_bytes;
    // device staging of the host-pointer entry points (b / x copies), grow-only
    void *stage;
    size_t stage_bytes;
    // tiles exact in INT8 or FP16 (counted on first use; n_exact_known = 0 before)
    int n_exact_known;
    long long n_exact;
    long long n_fp16_ok;       // tiles whose values lie within FP16's normal range
    long long n_exact_f16;     // tiles whose values FP16 reproduces exactly
};

// Position of entry k of row i in the slice whose payload starts at entry
// offset `off` (a multiple of 128), for values of ESZ bytes (8, 4, 2, 1; the
// index bytes use 1): chunk k / 8, 16-byte group of g = 16 / ESZ entries (at
// most 8) within the chunk, row i's g entries contiguous inside the group.
template <int ESZ>
__host__ __device__ __forceinline__ long long mf_slot(long long off, int k, int i)
{
    constexpr int g = ESZ >= 8 ? 2 : ESZ == 4 ? 4 : 8;
    const int kc = k & 7;
    return off + (long long)(k >> 3) * 128 + (kc / g) * (16 * g) + i * g + (kc % g);
}

// ---------------------------------------------------------------- helpers

#define MF_CUDA_TRY(expr)                                   \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) {                            \
            mf_set_last_cuda_error(_e, #expr, __FILE__, __LINE__); \
            return (_e == cudaErrorMemoryAllocation) ? MF_ERR_NOMEM : MF_ERR_CUDA; \
        }                                                   \
    } while (0)

void mf_set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line);

// device exclusive scans (scan.cu)
int mf_scan_i32_to_i32(const int *d_in, int *d_out, long long n, cudaStream_t s);   // out[0..n]
int mf_scan_i32_to_i64(const int *d_in, long long *d_out, long long n, cudaStream_t s);
int mf_scan_i64_to_i64(const long long *d_in, long long *d_out, long long n, cudaStream_t s);

// tile build (tile_build.cu)
int mf_build_tiles(mf_matrix_s *A, cudaStream_t s);

// solver (solver.cu)
int mf_solver_run(mf_matrix_s *A, const double *d_b, double *d_x, const mf_options *opt,
                  mf_report *rep, cudaStream_t s);
int mf_solver_multi_run(mf_matrix_s *A, int nrhs, const double *d_B, double *d_X, const mf_options *opt,
                        mf_report *reps, cudaStream_t s);
// Batched work items: interleave width of a group of g columns, and the
// estimated time of an item on one block: iterations x per-iteration work.
// Measured on one B200 (512-thread blocks, mixed CG, 8 columns), the
// per-iteration time of one block is set by the rows (the vector phases and
// the per-row gathers), not by the entries: a 5-point and a 27-point system of
// ~250,000 rows took the same time per row within 10 %; entries count as 1/64
// of a row.  Iterations are taken as n^0.4 (CG on these diffusion systems
// needs ~ side iterations: n^0.5 in 2D, n^0.33 in 3D).  The device queue's
// order, the team sizes and the split across GPUs (mf_batch_partition) all use it.
inline int mf_batch_width(int g) { return g >= 5 ? 8 : g >= 3 ? 4 : g == 2 ? 2 : 1; }
inline double mf_batch_item_cost(long long nnz, int n, int width)
{
    const double rows = (double)(n > 1 ? n : 1);
    return (rows + (double)nnz / 64.0) * (1.0 + 0.35 * (double)(width - 1)) * std::pow(rows, 0.4);
}
int mf_batch_create_impl(mf_batch_s **out, int nsys, mf_matrix_s *const *systems, const int *nrhs, cudaStream_t s);
int mf_batch_solve_impl(mf_batch_s *b, const double *const *Bd, double *const *Xd, const mf_options *opt,
                        mf_report *reps, int use_graph, cudaStream_t s);
int mf_batch_tune_impl(mf_batch_s *b, int precision, int iters, int *chosen, cudaStream_t s);
int mf_batch_configure_impl(mf_batch_s *b, int cap, int lb, cudaStream_t s);
void mf_batch_config_impl(const mf_batch_s *b, int *cap, int *lb);
void mf_batch_destroy_impl(mf_batch_s *b);
int mf_batch_schedule_impl(int nitems, const double *cost, const int *tilem, int grid, int *team, int *bptr,
                           int *blist, int *queue, int *nqueue);
int mf_spmv_run(mf_matrix_s *A, const double *d_x, double *d_y, int precision, cudaStream_t s,
                double *elapsed_ms);
int mf_spmv_tiles_run(mf_matrix_s *A, const double *d_x, double *d_y, int tile_prec, cudaStream_t s,
                      double *elapsed_ms);
int mf_solver_labels_run(mf_matrix_s *A, int *vis, int nseg);
int mf_spmm_run(mf_matrix_s *A, const double *d_X, double *d_Y, int tensor_cores, cudaStream_t s,
                double *elapsed_ms);
int mf_spmv_noalloc_run(mf_matrix_s *A, const double *d_x, double *d_y, int precision, cudaStream_t s);
int mf_ref_labels_run(const double *d_pold, const double *d_pnew, int nseg, int *d_vis,
                      cudaStream_t s);
void mf_solver_free_ws(mf_matrix_s *A);

// ------------------------------------------------------- device utilities
#ifdef __CUDACC__
__device__ __forceinline__ unsigned int mf_ld_acquire_u32(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned int mf_ld_relaxed_u32(const unsigned int *p)
{
    unsigned int v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void mf_red_release_add_u32(unsigned int *p, unsigned int v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void mf_red_relaxed_add_u32(unsigned int *p, unsigned int v)
{
    asm volatile("red.relaxed.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// 16-byte release store / acquire load (two 64-bit words) at gpu scope
__device__ __forceinline__ void mf_st_release_v2(unsigned long long *p, unsigned long long a, unsigned long long b)
{
    asm volatile("st.release.gpu.global.v2.b64 [%0], {%1, %2};" ::"l"(p), "l"(a), "l"(b) : "memory");
}
__device__ __forceinline__ void mf_st_relaxed_v2(unsigned long long *p, unsigned long long a, unsigned long long b)
{
    asm volatile("st.relaxed.gpu.global.v2.b64 [%0], {%1, %2};" ::"l"(p), "l"(a), "l"(b) : "memory");
}
__device__ __forceinline__ void mf_ld_acquire_v2(const unsigned long long *p, unsigned long long &a,
                                                 unsigned long long &b)
{
    asm volatile("ld.acquire.gpu.global.v2.b64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p) : "memory");
}
__device__ __forceinline__ void mf_ld_relaxed_v2(const unsigned long long *p, unsigned long long &a,
                                                 unsigned long long &b)
{
    asm volatile("ld.relaxed.gpu.global.v2.b64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p) : "memory");
}
__device__ __forceinline__ unsigned long long mf_globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mf_fence_acq_rel_gpu()
{
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
}
// streaming (evict-first) loads for the read-once matrix payload
__device__ __forceinline__ double mf_ld_stream(const double *p) { return __ldcs(p); }
__device__ __forceinline__ float mf_ld_stream(const float *p) { return __ldcs(p); }
__device__ __forceinline__ unsigned long long mf_ld_stream(const unsigned long long *p) { return __ldcs(p); }
#endif
