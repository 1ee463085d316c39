/*
 * millefeuille.h -- C ABI of the B200 (sm_100a) tile-grained mixed-precision
 * single-kernel CG / BiCGSTAB library (libmillefeuille.so).
 *
 * Plain pointers and sizes only.  Two layers:
 *
 *  1. Drop-in entry points with the reference's exact signatures
 *     (cg_solve_inc / cg_solve_sync / cg_solve_reduce, bicgstab /
 *     bicgstab_sync / bicgstab_inc, Tile_create-equivalent export).
 *  2. The native API: an opaque device-resident tiled matrix, mf_solve,
 *     mf_spmv, tile export for parity checks, and status codes.
 *
 * Every function returns or records an mf_status; nothing calls exit() or
 * traps.  Device spin-waits are bounded; a wait that runs out returns
 * MF_ERR_TIMEOUT.  One CUDA device per process thread (the current device);
 * handles are independent and may be used from different host threads.
 */
#ifndef MILLEFEUILLE_H
#define MILLEFEUILLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
typedef enum {
    MF_SUCCESS = 0,
    MF_ERR_INVALID = 1,        /* bad argument / malformed CSR */
    MF_ERR_CUDA = 2,           /* a CUDA runtime call failed */
    MF_ERR_NOMEM = 3,          /* device allocation failed */
    MF_ERR_TIMEOUT = 4,        /* a bounded device wait ran out */
    MF_ERR_UNSUPPORTED = 5,    /* input outside the supported envelope */
    MF_ERR_BREAKDOWN = 6,      /* a Krylov scalar became 0 / non-finite */
    MF_ERR_IO = 7,             /* matrix file could not be read */
    MF_ERR_NOT_BUILT = 8,      /* no CUDA device available */
    MF_ERR_CHECK = 9           /* bounds-checked build only: a kernel index failed its bounds check
                                  (the access was skipped; site, index and limit go to stderr) */
} mf_status;

const char *mf_status_string(int status);

/* ------------------------------------------------------ drop-in boundary */

/* Result record of the reference drivers (main-cg-mixed.cu:11-16). */
typedef struct {
    double time_ms;     /* solve time (CUDA events around the single launch) */
    int iterations;     /* iterations executed */
    double l2_norm;     /* ||A x - b|| / ||b|| computed in FP64 */
    double residual;    /* recursive ||r|| (absolute) */
} CgBenchResult;

/*
 * Replaces cg_solve_inc of main-cg-mixed.cu:2248 (mixed-precision single
 * kernel) in libmillefeuille.so, and cg_solve_inc of main-cg.cu:1110 (FP64;
 * main-cg calls it for nnz < 10,000, main-cg.cu:1727-1745) in
 * libmillefeuille_fp64.so, which is otherwise the same library: link the
 * library that matches the reference driver being replaced (mf_build_arch
 * names the variant; the FP64 one writes cg_performance.csv).
 * Same arguments and meaning: n is the row count already truncated
 * to a multiple of 16 by the caller, ori the original column count, x is
 * zeroed and returned, exactly max_iter iterations are run (the reference has
 * no convergence exit); iter, maxiter and threshold are ignored as in the
 * reference; a CSV row is appended to "cg_mixed_performance.csv" unless
 * skip_output.  Val_Low may be NULL (then (float)Val is used).
 */
void cg_solve_inc(int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x, double *b,
                  int n, int *iter, int maxiter, double threshold, char *filename, int nnzR,
                  int ori, int max_iter, CgBenchResult *bench_result, int skip_output);
/* Replaces cg_solve_sync of main-cg.cu:405 (FP64 single kernel). */
void cg_solve_sync(int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x, double *b,
                   int n, int *iter, int maxiter, double threshold, char *filename, int nnzR,
                   int ori, int max_iter, CgBenchResult *bench_result, int skip_output);
/* Replaces cg_solve_reduce of main-cg.cu:19 (FP64; the reference's multi-kernel
 * host loop becomes the same single persistent kernel here). */
void cg_solve_reduce(int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x, double *b,
                     int n, int *iter, int maxiter, double threshold, char *filename, int nnzR,
                     int ori, int max_iter, CgBenchResult *bench_result, int skip_output);
/*
 * Replaces bicgstab of main-bicg-mixed.cu:1355 (mixed-precision single kernel,
 * fixed 50 iterations, rhs overwritten with the row sums A*1 as the reference
 * does, x is the output).  Returns 0; prints "time_bicg=... ms" like the
 * reference and appends to "bicg_mixed_performance.csv".
 */
int bicgstab(int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x, int nnzR,
             char *filename, int n);
/* Replace bicgstab_sync / bicgstab_inc of main-bicg.cu:13,711 (FP64 single
 * kernel, fixed 50 iterations, rhs overwritten with row sums). */
int bicgstab_sync(int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x, int nnzR,
                  char *filename, int n);
int bicgstab_inc(int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x, int nnzR,
                 char *filename, int n);

/*
 * Replaces read_Dmatrix_32 (biio2.0/src/biio.h:153-194): reads a Matrix
 * Market (.mtx) or binary CSR (.cbd) file into 0-based CSR with the
 * reference's ordering (file order within a row, symmetric entries mirrored).
 * Arrays are allocated with malloc; free them with mf_free_host.
 */
int mf_read_matrix(const char *path, int *m, int *n, int *nnz, int **rowptr, int **colidx,
                   double **val, int *is_symmetric);
/* Writes binary CSR (.cbd, biio.h:74-97 layout). */
int mf_write_cbd(const char *path, int m, int n, int nnz, const int *rowptr, const int *colidx,
                 const double *val);
void mf_free_host(void *p);

/* ------------------------------------------------------------ native API */

typedef enum { MF_METHOD_CG = 0, MF_METHOD_BICGSTAB = 1 } mf_method;

typedef enum {
    MF_PREC_FP64 = 0,     /* all tiles FP64 ("same kernel in all-FP64") */
    MF_PREC_MIXED = 1,    /* default: FP32/FP16/INT8 tile products, FP64 dots/updates */
    MF_PREC_PARITY = 2    /* reference label rule and tile arithmetic (not numerically safe) */
} mf_precision;

typedef struct {
    int method;            /* mf_method */
    int precision;         /* mf_precision */
    double tol;            /* relative residual target ||b-Ax||/||b|| */
    int max_iter;          /* iteration cap */
    int fixed_iters;       /* 1: run exactly max_iter iterations (reference semantics) */
    int replace_every;     /* FP64 true-residual replacement period (0: only at convergence) */
    double demote_fp16;    /* mixed: column segment max|p| / max|p| below this -> FP16 tiles */
    double demote_int8;    /* mixed: ... below this -> scaled INT8 tiles */
    int use_lossless;      /* mixed: tiles exactly representable in a narrower type use it */
    double wait_timeout_s; /* bound on every device spin-wait */
    int blocks_per_sm;     /* 0: from occupancy */
    int threads_per_block; /* 0: default (512) */
    int x0_given;          /* 1: x holds the initial guess on entry (mf_solve: CG and BiCGSTAB, every
                              precision; mf_solve_multi and mf_batch_solve: X, every column; the
                              first residual r = b - A x is formed in FP64) */
    int l2_window;         /* 1 (default): keep the solver vectors in L2 with a persisting
                              access-policy window on the stream during the solve */
    int test_stall_barrier;/* test hook: 1 = the first grid barrier waits for one arrival that
                              never comes; the bounded wait runs out after wait_timeout_s and the
                              solve returns MF_ERR_TIMEOUT (no fault, the context stays usable) */
    double demote_min_fraction; /* mixed: narrower tiles are considered in an SpMV only when at least
                              this fraction of the operand's column segments fell below demote_fp16
                              of its maximum in the previous update (or of the tiles are exact in a
                              narrower type, for use_lossless); below it every tile runs FP32.
                              Default 0.125; 0 = always consider them */
    double relax_eta;      /* mixed CG (mf_solve): relaxed matvec precision.  Once the recursive
                              relative residual rho has fallen so far that relax_eta * tol / rho
                              exceeds a stored precision's rounding (2^-11 FP16, 2^-8 scaled
                              INT8, see relax_int8), the whole SpMV runs in it (inexact Krylov
                              relaxation; the FP64 residual replacement and the FP64 convergence
                              test keep the final accuracy).  0 = off */
    int relax_int8;        /* with relax_eta: the relaxed precision may go down to scaled INT8
                              (default 0: FP16 at most) */
    int test_check_limit;  /* test hook of the bounds-checked build (libmillefeuille_check.so), mf_solve
                              only: the kernels check the operand's gathered entries against this
                              length (rounded down to a multiple of 16) instead of the padded vector
                              length, so the check path runs without any out-of-bounds index.  0 = off;
                              the normal build ignores it */
} mf_options;

typedef struct {
    int status;            /* mf_status of the solve */
    int iterations;
    int converged;
    double relres_true;    /* FP64 ||b - A x|| / ||b|| at exit (on the GPU) */
    double relres_rec;     /* recursive residual ratio at exit */
    double residual;       /* recursive ||r|| (absolute) */
    double time_ms;        /* kernel time (CUDA events on the launch stream) */
    int replacements;      /* FP64 residual replacements performed */
    int grid_blocks;       /* persistent grid size */
    int threads_per_block;
    long long tile_uses[4];/* tile-products executed per precision: FP64, FP32, FP16, INT8 */
    long long tiles_skipped;
    long long nnz_uses[4]; /* matrix entries streamed per precision (same order); the FP64
                              residual-replacement SpMVs are not included */
    double phase_ms[6];    /* block 0's wall time split: SpMV phases, first vector update,
                              direction update, barriers + reductions, FP64 residual replacement;
                              [5]: of the barrier time, block 0 spinning for the other blocks */
    double host_ms[4];     /* mf_solve's host-side wall time: [0] staging buffer and H2D copy of b
                              enqueued (host pointers), [1] solver state zeroed and L2 window set,
                              [2] launch until the results are read back (includes the kernel),
                              [3] D2H copy of x and the closing synchronisation (host pointers) */
} mf_report;

void mf_options_default(mf_options *opt);

typedef struct mf_matrix_s *mf_matrix;

typedef struct {
    int n_rows, n_cols;
    long long nnz;
    int tilem, tilen, tilenum;
    int csrsize, csrptrlen, cnt_non_new, rowblkblock;
    int nseg;               /* solver slices */
    long long slice_entries;/* padded solver entries */
    double build_ms;        /* GPU tiling + encoding time */
    int device;             /* CUDA device the handle's memory lives on (current at create) */
} mf_matrix_info;

/*
 * Build a device-resident tiled matrix from 0-based CSR (n_rows rows; rows are
 * NOT truncated here).  Pointers are host pointers unless device_ptrs != 0.
 * val_low may be NULL ((float)val is used).  The GPU csr2block is bit-exact to
 * Tile_create (csr2block.h:267-422).  stream may be NULL (default stream).
 */
int mf_matrix_create(mf_matrix *out, int n_rows, int n_cols, long long nnz, const int *rowptr,
                     const int *colidx, const double *val, const float *val_low, int device_ptrs,
                     void *stream);
int mf_matrix_destroy(mf_matrix A);
int mf_matrix_get_info(mf_matrix A, mf_matrix_info *info);

/*
 * Copy one reference-layout array to host memory (for parity checks).  Names:
 * tile_ptr, tile_columnidx, tile_nnz, blknnz, csr_offset, csrptr_offset,
 * ptroffset1, ptroffset2, val, val_low, col, ptr, nonzero_row_new,
 * blockrowid_new, blockcsr_ptr_new, tile_rowidx, block_signal,
 * blkcoostylerowidx, colstart, colstop, val_f16, val_i8_ref, val_i8, i8_scale.
 * bytes must equal the array size; mf_tile_array_bytes reports it.
 */
int mf_tile_array_bytes(mf_matrix A, const char *name, size_t *bytes);
int mf_tile_export(mf_matrix A, const char *name, void *host_dst, size_t bytes);

/*
 * Solve A x = b (or with nrhs=1 only in this version).  b and x are host
 * pointers unless device_ptrs != 0; with host pointers the copies are part of
 * the call.  report may be NULL.
 */
int mf_solve(mf_matrix A, const double *b, double *x, const mf_options *opt, mf_report *report,
             int device_ptrs, void *stream);

/*
 * Solve A X = B for nrhs right-hand sides (CG; MF_PREC_FP64 or MF_PREC_MIXED).
 * B and X hold nrhs vectors of n_rows doubles one after another; host
 * pointers unless device_ptrs != 0.  Up to 8 columns run in one persistent
 * launch (every matrix entry read once per SpMV for all of them, one grid sync
 * for all of them); each column has its own alpha / beta, convergence test
 * and FP64 true-residual check.  reports (nullable) receives nrhs records
 * (time_ms and replacements are those of the column's launch).  nrhs == 1 is
 * mf_solve.  No counterpart in the reference (one right-hand side per call).
 */
int mf_solve_multi(mf_matrix A, int nrhs, const double *B, double *X, const mf_options *opt,
                   mf_report *reports, int device_ptrs, void *stream);

/*
 * Batched solves: many independent square systems (each an mf_matrix on the
 * current device) with nrhs[k] right-hand sides each, in ONE persistent launch.
 * Work items are (system, up to `cap` right-hand sides).  Items far above a
 * fair share of the launch are solved by teams of 512-thread blocks on a host
 * list schedule; the rest sit in a device work queue, largest estimated cost
 * first, and a block takes the next one and solves it alone (CG, FP64 or
 * mixed; block-level syncs).  One cooperative launch of one or two blocks per
 * SM.  No counterpart in the reference (one system per call).
 *
 * mf_batch_create  keeps the handles' pointers (the matrices must outlive the
 *                  batch) and sizes the work items (cap 8, one block per SM).
 * mf_batch_tune    picks the right-hand sides per item and the blocks per SM
 *                  ((8,1), (4,1), (2,1), (4,2), (2,2)) by timing `iters` fixed
 *                  iterations of the real batch (two blocks per SM count 15 %
 *                  slower than timed: the short probe favours them over a
 *                  full solve's tail of long items); *chosen_cap (nullable) gets
 *                  the right-hand sides per item (grid_blocks in the reports
 *                  shows the blocks).
 * mf_batch_configure sets the right-hand sides per item (1, 2, 4 or 8) and the
 *                  blocks per SM (1, or 2 for items of up to 4 columns where two
 *                  blocks fit) without timing runs, e.g. to reuse what
 *                  mf_batch_tune chose for a batch of the same shapes (new
 *                  values, same sizes); MF_ERR_INVALID for other pairs.
 * mf_batch_config  reads the current pair.
 * mf_batch_solve   B[k] / X[k]: DEVICE arrays of nrhs[k] x n_k doubles (one
 *                  vector after another).  reports (nullable): sum(nrhs)
 *                  records, system by system; time_ms is the whole batch's;
 *                  phase_ms[0] / [1]: the column's work item's start and end
 *                  in ms after the launch's first item start, phase_ms[2]: the
 *                  blocks that solved it.
 *                  use_graph != 0: the enqueue sequence (interleave, queue
 *                  reset, launch, de-interleave) is captured into a CUDA graph
 *                  on first use and replayed while the pointers and options stay
 *                  the same.  stream NULL: the batch's own stream.
 */
typedef struct mf_batch_s *mf_batch;
int mf_batch_create(mf_batch *out, int nsys, const mf_matrix *systems, const int *nrhs, void *stream);
int mf_batch_tune(mf_batch b, int precision, int iters, int *chosen_cap, void *stream);
int mf_batch_configure(mf_batch b, int cap, int blocks_per_sm, void *stream);
int mf_batch_config(mf_batch b, int *cap, int *blocks_per_sm);
int mf_batch_solve(mf_batch b, const double *const *B, double *const *X, const mf_options *opt,
                   mf_report *reports, int use_graph, void *stream);
int mf_batch_destroy(mf_batch b);

/*
 * The team sizes and list schedule a batch launch of `grid` blocks uses for
 * items of estimated cost cost[t] and tilem[t] tile-rows (host only; for
 * inspection and tests).  team[t] (nitems): blocks solving item t (1: queue
 * item).  bptr (grid + 1) and blist (2 ints per entry: item, rank in its team;
 * at most sum(team) entries): block b's ordered team entries are
 * blist[2*bptr[b] .. 2*bptr[b+1]).  queue (nitems): the queue items, largest
 * cost first; *nqueue their count.  No counterpart in the reference.
 */
int mf_batch_schedule(int nitems, const double *cost, const int *tilem, int grid, int *team, int *bptr,
                      int *blist, int *queue, int *nqueue);

/*
 * Split of a batch's systems over nparts GPUs (one process per GPU, each with
 * its own mf_batch of the systems it owns; no collective on the data path).
 * Greedy longest-processing-time over whole systems, by decreasing estimated
 * cost -- the sum over the system's work items of groups of <= cap columns
 * (cap 1..8; <= 0 means 8) of (n + nnz / 64) * (1 + 0.35 (width - 1)) * n^0.4, the cost
 * the work queue orders by -- each to the least-loaded part so far; ties go to
 * the lower index.  part[k] (nsys ints) gets system k's part; load (nullable,
 * nparts doubles) each part's total cost.  Host only, deterministic: every rank
 * computes the same split.  No counterpart in the reference.
 */
int mf_batch_partition(int nsys, const int *n, const long long *nnz, const int *nrhs, int cap, int nparts,
                       int *part, double *load);

/* y = A x with the tile kernel.  precision: MF_PREC_FP64 or MF_PREC_MIXED
 * (MIXED here means every tile in FP32).  elapsed_ms (nullable) gets the kernel time. */
int mf_spmv(mf_matrix A, const double *x, double *y, int precision, int device_ptrs,
            void *stream, double *elapsed_ms);

/*
 * y = A x like mf_spmv, but the call allocates no memory (no cudaMalloc /
 * cudaFree, no host staging).  No counterpart in the reference: its
 * entry points allocate and free device memory on every call.  For callers
 * that must not allocate -- code that runs with the device memory already
 * handed to another allocator, or inside a latency-critical loop where an
 * allocation's implicit device synchronisation is not acceptable.
 *
 *  - x and y are device pointers (n_cols and n_rows doubles); precision is
 *    MF_PREC_FP64 or MF_PREC_MIXED (every tile in FP32), as for mf_spmv.
 *  - The call is asynchronous on `stream` (NULL: default stream); y is ready
 *    when the stream reaches that point.
 *  - Scratch: the padded copy of x lives in a fixed device buffer compiled
 *    into the library, MF_SPMV_NOALLOC_MAX_LEN doubles (16 MB per device).  Matrices whose padded vector length,
 *    16 * ceil(max(n_rows, n_cols) / 16), exceeds it are rejected with
 *    MF_ERR_UNSUPPORTED before anything is launched.
 *  - Nothing has to start at zero: each call writes every scratch entry the
 *    kernel reads (x, then zeros up to the padded length).
 *  - The current device must be the one the matrix was created on
 *    (mf_matrix_info.device); otherwise the call returns MF_ERR_INVALID.
 *  - The first call on a device looks the buffer up (cudaGetSymbolAddress,
 *    which may load the library's device code); make that first call before
 *    any stream capture.  Later calls only issue a copy, a memset and the
 *    kernel.  The address is kept for the life of the loaded library: a
 *    cudaDeviceReset in the caller's process unloads the device code and
 *    leaves it stale, so after a reset the library must be unloaded and
 *    loaded again before this entry point is called.
 *  - One buffer per device is shared by all handles and threads: calls on
 *    the same device must not overlap in time (issue them on one stream, or
 *    order the streams), otherwise they race on the scratch.
 */
#define MF_SPMV_NOALLOC_MAX_LEN (1 << 21)
int mf_spmv_noalloc(mf_matrix A, const double *x, double *y, int precision, void *stream);

/* ------------------------------------------------- differentiation support
 * No counterpart in the reference (it has no differentiation).  For
 * A x = b and a loss L(x): lambda = A^-T dL/dx (an adjoint solve: the same
 * solver on A for symmetric A, on a transposed handle otherwise), then
 * dL/db = lambda and dL/dA = -lambda x^T on A's stored pattern.
 */

/* grad_val[e] = -sum_k lambda[k*n_rows + i] * x[k*n_cols + j] for every stored
 * entry e = (i, j) of A, in the order of the CSR A was created from (entries of
 * rows [0, n_rows)); nrhs right-hand sides stored one after another.  Pointers
 * are host pointers unless device_ptrs != 0.  Deterministic. */
int mf_value_grad(mf_matrix A, int nrhs, const double *lambda, const double *x, double *grad_val,
                  int device_ptrs, void *stream);

/* A handle for A^T (n_cols x n_rows), built from A's CSR; rows of A^T keep
 * A's row order (stable, deterministic).  Destroy it with mf_matrix_destroy. */
int mf_matrix_create_transposed(mf_matrix *out, mf_matrix A, void *stream);

/* Test hook: segment labels of the reference rule for (p_old, p_new) device or
 * host arrays of length nseg*16; codes as d_vis (0 FP64, 4 FP32, 3 FP16, 2 INT8,
 * 1 bypass).  Runs the same device classifier the parity-mode solver uses. */
int mf_debug_ref_labels(const double *p_old, const double *p_new, int nseg, int *vis,
                        int device_ptrs);

/* Test hook: y = A x with every tile's stored values in one precision:
 * tile_prec 0 FP64, 1 FP32 (Val_Low), 2 FP16 (round-to-nearest of the FP32
 * value, the reference encoder's half), 3 INT8 with this library's per-tile
 * scale.  The stored value is widened to FP64 and multiplied with the FP64 x;
 * row sums are FP64 in the slice walk's entry order (tile by tile, payload
 * order within a tile).  Host pointers unless device_ptrs != 0; synchronous.
 * No counterpart in the reference (its FP16 / INT8 products run only inside
 * the solver, in half / int8 arithmetic). */
int mf_debug_spmv_tiles(mf_matrix A, const double *x, double *y, int tile_prec, int device_ptrs);

/* Experiment hook: Y = A X for 8 right-hand sides (columns one after another,
 * n_cols / n_rows doubles each) with every tile's values stored in FP16.
 * tensor_cores = 0: the solver's CUDA-core arithmetic (FP16 value widened to
 * FP64 against the FP64 X); 1: each 16 x 16 tile densified in shared memory
 * from the sparse payload and multiplied with the FP16-rounded 16 x 8 block
 * of X by one mma.sync.m16n8k16 per tile (FP32 accumulation).  elapsed_ms
 * (nullable): the kernel's time.  Host pointers unless device_ptrs != 0.
 * No counterpart in the reference. */
int mf_debug_spmm(mf_matrix A, const double *X, double *Y, int tensor_cores, int device_ptrs,
                  double *elapsed_ms);

/* Test hook: the labels the last mf_solve on A in MF_PREC_PARITY left for the
 * next SpMV's operand p (d_vis codes: 0 FP64, 4 FP32, 3 FP16, 2 INT8, 1
 * bypass), one per column segment (main-cg-mixed.cu:1323-1370 computes them);
 * nseg <= max(tilem, tilen).  Undefined after solves in the other precisions. */
int mf_debug_solver_labels(mf_matrix A, int *vis, int nseg);

/* Test hook: the full report (mf_report) of the calling thread's last
 * drop-in solve (cg_solve_inc / _sync / _reduce, bicgstab / _sync / _inc), so a
 * caller of the reference's entry points can see which precision ran
 * (tile_uses).  No counterpart in the reference. */
int mf_dropin_last_report(mf_report *out);

/* Library build identity (e.g. "sm_100a"). */
const char *mf_build_arch(void);

#ifdef __cplusplus
}
#endif
#endif /* MILLEFEUILLE_H */
