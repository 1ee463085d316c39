// api.cu -- the C ABI of libmillefeuille.so (declared in include/millefeuille.h).
#include "mf_internal.cuh"

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

static thread_local char g_last_err[512];

namespace {
// NVTX range around a C-ABI call, so profilers (ncu --nvtx, Nsight Systems)
// can attribute kernels to the call that launched them; free without a tool.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};
}  // namespace

void mf_set_last_cuda_error(cudaError_t e, const char *what, const char *file, int line)
{
    snprintf(g_last_err, sizeof(g_last_err), "%s (%s) at %s:%d: %s", cudaGetErrorName(e), what, file, line,
             cudaGetErrorString(e));
}

#define MF_TRY(expr)                        \
    do {                                    \
        int _rc = (expr);                   \
        if (_rc != MF_SUCCESS) return _rc;  \
    } while (0)

extern "C" {

const char *mf_status_string(int status)
{
    switch (status) {
    case MF_SUCCESS: return "success";
    case MF_ERR_INVALID: return "invalid argument or malformed CSR";
    case MF_ERR_CUDA: return g_last_err[0] ? g_last_err : "CUDA runtime error";
    case MF_ERR_NOMEM: return "device allocation failed";
    case MF_ERR_TIMEOUT: return "a bounded device wait ran out (grid barrier timeout)";
    case MF_ERR_UNSUPPORTED: return "input outside the supported envelope";
    case MF_ERR_BREAKDOWN: return "Krylov breakdown (zero or non-finite scalar)";
    case MF_ERR_IO: return "matrix file could not be read";
    case MF_ERR_NOT_BUILT: return "no CUDA device available";
    case MF_ERR_CHECK: return "a kernel index failed its bounds check (bounds-checked build)";
    default: return "unknown status";
    }
}

#if defined(MF_CHECK)
const char *mf_build_arch(void) { return "sm_100a (bounds-checked)"; }
#elif defined(MF_CG_INC_FP64)
const char *mf_build_arch(void) { return "sm_100a (cg_solve_inc: FP64, main-cg.cu)"; }
#else
const char *mf_build_arch(void) { return "sm_100a"; }
#endif

void mf_options_default(mf_options *o)
{
    memset(o, 0, sizeof(*o));
    o->method = MF_METHOD_CG;
    o->precision = MF_PREC_MIXED;
    o->tol = 1e-8;
    o->max_iter = 10000;
    o->fixed_iters = 0;
    o->replace_every = 50;
    o->demote_fp16 = 1.0 / 8192.0;     // 2^-13: FP16 rounding no larger than FP32's on the largest entries
    o->demote_int8 = 1.0 / 65536.0;    // 2^-16: likewise for per-tile scaled INT8
    o->use_lossless = 1;
    o->wait_timeout_s = 10.0;
    o->blocks_per_sm = 0;
    o->threads_per_block = 0;
    o->x0_given = 0;
    o->l2_window = 1;
    o->test_stall_barrier = 0;
    o->demote_min_fraction = 0.125;
    o->relax_eta = 0.0;
    o->relax_int8 = 0;
}

void mf_free_host(void *p) { free(p); }

}  // extern "C"

// ------------------------------------------------------------------ matrices
namespace {

__global__ void k_check_rowptr(const int *rowptr, int n, long long nnz, int *err)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int a = rowptr[i], b = rowptr[i + 1];
        if (a < 0 || b < a || (long long)b > nnz) atomicExch(err, MF_ERR_INVALID);
    }
}

void free_matrix(mf_matrix_s *A)
{
    mf_solver_free_ws(A);
    void *ptrs[] = {A->d_rowptr, A->d_colidx, A->d_val, A->d_val_low, A->d_tile_ptr, A->d_tile_columnidx,
                    A->d_csr_offset, A->d_csrptr_offset, A->d_tval, A->d_tval_low, A->d_tcol, A->d_tptr,
                    A->d_nonzero_row_new, A->d_tile_rowidx, A->d_block_signal, A->d_blockrowid_new,
                    A->d_blockcsr_ptr_new, A->d_rb_idx, A->d_rb_start, A->d_rb_stop, A->d_val_f16,
                    A->d_val_i8_ref, A->d_val_i8, A->d_i8_scale, A->d_tile_caps, A->d_seg_ptr, A->d_seg_tile0,
                    A->d_seg_off, A->d_seg_hdr, A->d_seg_tile, A->d_seg_kp, A->d_seg_rowlen, A->d_meta, A->d_v64, A->d_v32, A->d_v16,
                    A->d_v8, A->d_v8ref, A->d_row_cost};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (A->stage) cudaFree(A->stage);
    delete A;
}

// Device staging of a host-pointer call (copies of b and x), kept in the handle
// and grown when a call needs more, so a solve allocates and frees nothing once
// warm (a stream-ordered allocation per call was returned to the driver at the
// call's closing synchronisation and mapped again on the next call).
int stage_get(mf_matrix_s *A, size_t bytes, double **out)
{
    if (A->stage_bytes < bytes) {
        if (A->stage) cudaFree(A->stage);
        A->stage = nullptr;
        A->stage_bytes = 0;
        MF_CUDA_TRY(cudaMalloc(&A->stage, bytes));
        A->stage_bytes = bytes;
    }
    *out = (double *)A->stage;
    return MF_SUCCESS;
}

int device_ready()
{
    int nd = 0;
    if (cudaGetDeviceCount(&nd) != cudaSuccess || nd < 1) {
        cudaGetLastError();
        return MF_ERR_NOT_BUILT;
    }
    return MF_SUCCESS;
}

}  // namespace

extern "C" int mf_matrix_create(mf_matrix *out, int n_rows, int n_cols, long long nnz, const int *rowptr,
                                const int *colidx, const double *val, const float *val_low, int device_ptrs,
                                void *stream)
{
    NvtxRange nvtx_range("mf_matrix_create");
    if (!out || n_rows < 0 || n_cols < 0 || nnz < 0 || !rowptr || (nnz > 0 && (!colidx || !val)))
        return MF_ERR_INVALID;
    if (nnz >= (1LL << 31)) return MF_ERR_UNSUPPORTED;
    *out = nullptr;
    MF_TRY(device_ready());
    cudaStream_t s = (cudaStream_t)stream;
    mf_matrix_s *A = new mf_matrix_s();
    memset(A, 0, sizeof(*A));
    MF_CUDA_TRY(cudaGetDevice(&A->dev));
    A->n_rows = n_rows;
    A->n_cols = n_cols;
    const cudaMemcpyKind kind = device_ptrs ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    int rc = MF_SUCCESS;
    auto fail = [&](int code) { free_matrix(A); return code; };
    if (cudaMalloc((void **)&A->d_rowptr, (size_t)(n_rows + 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc((void **)&A->d_colidx, (size_t)std::max<long long>(nnz, 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc((void **)&A->d_val, (size_t)std::max<long long>(nnz, 1) * sizeof(double)) != cudaSuccess)
        return fail(MF_ERR_NOMEM);
    if (val_low && cudaMalloc((void **)&A->d_val_low, (size_t)std::max<long long>(nnz, 1) * sizeof(float)) != cudaSuccess)
        return fail(MF_ERR_NOMEM);
    if (cudaMemcpyAsync(A->d_rowptr, rowptr, (size_t)(n_rows + 1) * sizeof(int), kind, s) != cudaSuccess ||
        (nnz > 0 && cudaMemcpyAsync(A->d_colidx, colidx, (size_t)nnz * sizeof(int), kind, s) != cudaSuccess) ||
        (nnz > 0 && cudaMemcpyAsync(A->d_val, val, (size_t)nnz * sizeof(double), kind, s) != cudaSuccess) ||
        (val_low && nnz > 0 &&
         cudaMemcpyAsync(A->d_val_low, val_low, (size_t)nnz * sizeof(float), kind, s) != cudaSuccess))
        return fail(MF_ERR_CUDA);
    int *d_err = nullptr;
    if (cudaMalloc((void **)&d_err, sizeof(int)) != cudaSuccess) return fail(MF_ERR_NOMEM);
    cudaMemsetAsync(d_err, 0, sizeof(int), s);
    if (n_rows > 0) k_check_rowptr<<<(n_rows + 255) / 256, 256, 0, s>>>(A->d_rowptr, n_rows, nnz, d_err);
    int h_err = 0;
    cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) { cudaFree(d_err); return fail(MF_ERR_CUDA); }
    cudaFree(d_err);
    if (h_err) return fail(h_err);
    rc = mf_build_tiles(A, s);
    if (rc != MF_SUCCESS) return fail(rc);
    *out = A;
    return MF_SUCCESS;
}

extern "C" int mf_matrix_destroy(mf_matrix A)
{
    if (!A) return MF_ERR_INVALID;
    free_matrix(A);
    return MF_SUCCESS;
}

extern "C" int mf_matrix_get_info(mf_matrix A, mf_matrix_info *info)
{
    if (!A || !info) return MF_ERR_INVALID;
    info->n_rows = A->n_rows;
    info->n_cols = A->n_cols;
    info->nnz = A->nnz;
    info->tilem = A->tilem;
    info->tilen = A->tilen;
    info->tilenum = A->tilenum;
    info->csrsize = A->csrsize;
    info->csrptrlen = A->csrptrlen;
    info->cnt_non_new = A->cnt_non_new;
    info->rowblkblock = A->rowblkblock;
    info->nseg = A->nseg;
    info->slice_entries = A->slice_entries;
    info->build_ms = A->build_ms;
    info->device = A->dev;
    return MF_SUCCESS;
}

namespace {
struct ArrayRef {
    const void *ptr;
    size_t bytes;
};

ArrayRef lookup(mf_matrix_s *A, const char *name)
{
    const size_t T = (size_t)A->tilenum, M = (size_t)A->tilem, Z = (size_t)A->csrsize;
    const std::string s(name);
    if (s == "tile_ptr") return {A->d_tile_ptr, (M + 1) * 4};
    if (s == "tile_columnidx") return {A->d_tile_columnidx, T * 4};
    if (s == "tile_nnz" || s == "blknnz" || s == "csr_offset") return {A->d_csr_offset, (T + 1) * 4};
    if (s == "csrptr_offset") return {A->d_csrptr_offset, (T + 1) * 4};
    if (s == "ptroffset1") return {A->d_csr_offset, T * 4};
    if (s == "ptroffset2") return {A->d_csrptr_offset, T * 4};
    if (s == "val") return {A->d_tval, Z * 8};
    if (s == "val_low") return {A->d_tval_low, Z * 4};
    if (s == "col") return {A->d_tcol, Z};
    if (s == "ptr") return {A->d_tptr, (size_t)A->csrptrlen};
    if (s == "nonzero_row_new") return {A->d_nonzero_row_new, (T + 1) * 4};
    if (s == "blockrowid_new") return {A->d_blockrowid_new, (size_t)A->cnt_non_new + 1};
    if (s == "blockcsr_ptr_new") return {A->d_blockcsr_ptr_new, (size_t)A->cnt_non_new + 1};
    if (s == "tile_rowidx") return {A->d_tile_rowidx, T * 4};
    if (s == "block_signal") return {A->d_block_signal, (M + 4) * 4};
    if (s == "blkcoostylerowidx") return {A->d_rb_idx, (size_t)A->rowblkblock * 4};
    if (s == "colstart") return {A->d_rb_start, (size_t)A->rowblkblock * 4};
    if (s == "colstop") return {A->d_rb_stop, (size_t)A->rowblkblock * 4};
    if (s == "val_f16") return {A->d_val_f16, Z * 2};
    if (s == "val_i8_ref") return {A->d_val_i8_ref, Z};
    if (s == "val_i8") return {A->d_val_i8, Z};
    if (s == "i8_scale") return {A->d_i8_scale, T * 4};
    if (s == "tile_caps") return {A->d_tile_caps, T};
    if (s == "seg_ptr") return {A->d_seg_ptr, (M + 1) * 4};
    if (s == "seg_kp") return {A->d_seg_kp, (size_t)A->nseg * 4};
    if (s == "seg_rowlen") return {A->d_seg_rowlen, (size_t)A->nseg * 16 * 2};
    if (s == "seg_off") return {A->d_seg_off, ((size_t)A->nseg + 1) * 8};
    if (s == "meta") return {A->d_meta, (size_t)A->slice_entries};
    if (s == "v64") return {A->d_v64, (size_t)A->slice_entries * 8};
    if (s == "v32") return {A->d_v32, (size_t)A->slice_entries * 4};
    if (s == "seg_hdr") return {A->d_seg_hdr, (size_t)A->nseg * 16};
    return {nullptr, 0};
}
}  // namespace

namespace {
// Tile_create quirk (csr2block.h:237,252 with utils.h:52-53): when the last
// tile-row holds a single row, exclusive_scan_char(ptr, 1) returns without
// zeroing, so the row "start" keeps the row's count, the row-by-row copy copies
// nothing and that tile-row's payload stays zero.  The device arrays keep the
// true layout (the solver needs it); exported copies restate the quirk.
int restate_one_row_quirk(mf_matrix_s *A, const char *name, void *dst)
{
    if (A->tilem == 0 || A->n_rows - (A->tilem - 1) * MF_BS != 1) return MF_SUCCESS;
    const std::string s(name);
    static const char *payload[] = {"val", "val_low", "col", "val_f16", "val_i8_ref", "val_i8"};
    bool is_payload = false;
    for (const char *p : payload) is_payload |= (s == p);
    if (!is_payload && s != "ptr" && s != "i8_scale") return MF_SUCCESS;
    int t0 = 0, t1 = 0;
    MF_CUDA_TRY(cudaMemcpy(&t0, A->d_tile_ptr + A->tilem - 1, sizeof(int), cudaMemcpyDeviceToHost));
    MF_CUDA_TRY(cudaMemcpy(&t1, A->d_tile_ptr + A->tilem, sizeof(int), cudaMemcpyDeviceToHost));
    if (t1 <= t0) return MF_SUCCESS;
    std::vector<int> off((size_t)(t1 - t0 + 1));
    MF_CUDA_TRY(cudaMemcpy(off.data(), A->d_csr_offset + t0, off.size() * sizeof(int), cudaMemcpyDeviceToHost));
    if (is_payload) {
        size_t es = (s == "val") ? 8 : (s == "val_low") ? 4 : (s == "val_f16") ? 2 : 1;
        memset((char *)dst + (size_t)off[0] * es, 0, (size_t)(off.back() - off[0]) * es);
    } else if (s == "i8_scale") {
        memset((float *)dst + t0, 0, (size_t)(t1 - t0) * sizeof(float));
    } else {   // ptr: one entry per tile of that tile-row (csrptr_offset = t0*16 + (t-t0))
        unsigned char *p = (unsigned char *)dst;
        for (int t = t0; t < t1; t++) p[(size_t)t0 * MF_BS + (t - t0)] = (unsigned char)(off[t - t0 + 1] - off[t - t0]);
    }
    return MF_SUCCESS;
}
}  // namespace

extern "C" int mf_tile_array_bytes(mf_matrix A, const char *name, size_t *bytes)
{
    if (!A || !name || !bytes) return MF_ERR_INVALID;
    ArrayRef r = lookup(A, name);     // every known array is allocated (>= 1 element)
    if (!r.ptr) return MF_ERR_INVALID;
    *bytes = r.bytes;
    return MF_SUCCESS;
}

extern "C" int mf_tile_export(mf_matrix A, const char *name, void *host_dst, size_t bytes)
{
    if (!A || !name) return MF_ERR_INVALID;
    ArrayRef r = lookup(A, name);
    if (!r.ptr) return MF_ERR_INVALID;
    if (bytes != r.bytes) return MF_ERR_INVALID;
    if (bytes == 0) return MF_SUCCESS;
    MF_CUDA_TRY(cudaMemcpy(host_dst, r.ptr, bytes, cudaMemcpyDeviceToHost));
    return restate_one_row_quirk(A, name, host_dst);
}

extern "C" int mf_solve(mf_matrix A, const double *b, double *x, const mf_options *opt, mf_report *report,
                        int device_ptrs, void *stream)
{
    NvtxRange nvtx_range("mf_solve");
    if (!A || !b || !x) return MF_ERR_INVALID;
    mf_options o;
    if (opt) o = *opt; else mf_options_default(&o);
    if (!(o.tol >= 0.0) || o.max_iter < 0) return MF_ERR_INVALID;
    if (A->n_rows != A->n_cols && A->n_cols < A->n_rows) return MF_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nb = (size_t)A->n_rows * sizeof(double);
    const double *db = b;
    double *dx = x;
    double *tmp = nullptr;
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    if (!device_ptrs) {
        MF_TRY(stage_get(A, 2 * nb + 16, &tmp));
        MF_CUDA_TRY(cudaMemcpyAsync(tmp, b, nb, cudaMemcpyHostToDevice, s));
        db = tmp;
        dx = tmp + A->n_rows;
        if (o.x0_given) MF_CUDA_TRY(cudaMemcpyAsync(dx, x, nb, cudaMemcpyHostToDevice, s));
    }
    const auto t1 = clk::now();
    int rc = mf_solver_run(A, db, dx, &o, report, s);
    const auto t2 = clk::now();
    if (!device_ptrs) {
        cudaMemcpyAsync(x, dx, nb, cudaMemcpyDeviceToHost, s);
        MF_CUDA_TRY(cudaStreamSynchronize(s));
    }
    if (report) {
        report->host_ms[0] = std::chrono::duration<double, std::milli>(t1 - t0).count();
        report->host_ms[3] = std::chrono::duration<double, std::milli>(clk::now() - t2).count();
    }
    return rc;
}

extern "C" int mf_solve_multi(mf_matrix A, int nrhs, const double *B, double *X, const mf_options *opt,
                              mf_report *reports, int device_ptrs, void *stream)
{
    NvtxRange nvtx_range("mf_solve_multi");
    if (!A || !B || !X || nrhs < 1) return MF_ERR_INVALID;
    if (A->n_rows != A->n_cols) return MF_ERR_INVALID;
    mf_options o;
    if (opt) o = *opt;
    else mf_options_default(&o);
    if (nrhs == 1) {
        // one column: the single-column kernel
        return mf_solve(A, B, X, &o, reports, device_ptrs, stream);
    }
    cudaStream_t s = (cudaStream_t)stream;
    const size_t bytes = (size_t)nrhs * A->n_rows * sizeof(double);
    const double *dB = B;
    double *dX = X, *tmp = nullptr;
    if (!device_ptrs) {
        MF_TRY(stage_get(A, 2 * bytes, &tmp));
        MF_CUDA_TRY(cudaMemcpyAsync(tmp, B, bytes, cudaMemcpyHostToDevice, s));
        dB = tmp;
        dX = tmp + (size_t)nrhs * A->n_rows;
        if (o.x0_given) MF_CUDA_TRY(cudaMemcpyAsync(dX, X, bytes, cudaMemcpyHostToDevice, s));
    }
    int rc = mf_solver_multi_run(A, nrhs, dB, dX, &o, reports, s);
    if (!device_ptrs) {
        cudaMemcpyAsync(X, dX, bytes, cudaMemcpyDeviceToHost, s);
        MF_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return rc;
}

extern "C" int mf_batch_create(mf_batch *out, int nsys, const mf_matrix *systems, const int *nrhs, void *stream)
{
    if (!out || nsys < 1 || !systems || !nrhs) return MF_ERR_INVALID;
    *out = nullptr;
    MF_TRY(device_ready());
    return mf_batch_create_impl(out, nsys, systems, nrhs, (cudaStream_t)stream);
}

extern "C" int mf_batch_tune(mf_batch b, int precision, int iters, int *chosen_cap, void *stream)
{
    if (!b || iters < 1 || (precision != MF_PREC_FP64 && precision != MF_PREC_MIXED)) return MF_ERR_INVALID;
    return mf_batch_tune_impl(b, precision, iters, chosen_cap, (cudaStream_t)stream);
}

extern "C" int mf_batch_configure(mf_batch b, int cap, int blocks_per_sm, void *stream)
{
    if (!b) return MF_ERR_INVALID;
    return mf_batch_configure_impl(b, cap, blocks_per_sm, (cudaStream_t)stream);
}

extern "C" int mf_batch_config(mf_batch b, int *cap, int *blocks_per_sm)
{
    if (!b) return MF_ERR_INVALID;
    mf_batch_config_impl(b, cap, blocks_per_sm);
    return MF_SUCCESS;
}

extern "C" int mf_batch_solve(mf_batch b, const double *const *B, double *const *X, const mf_options *opt,
                              mf_report *reports, int use_graph, void *stream)
{
    NvtxRange nvtx_range("mf_batch_solve");
    if (!b || !B || !X) return MF_ERR_INVALID;
    mf_options o;
    if (opt) o = *opt;
    else mf_options_default(&o);
    return mf_batch_solve_impl(b, B, X, &o, reports, use_graph, (cudaStream_t)stream);
}

extern "C" int mf_batch_destroy(mf_batch b)
{
    if (!b) return MF_ERR_INVALID;
    mf_batch_destroy_impl(b);
    return MF_SUCCESS;
}

extern "C" int mf_batch_schedule(int nitems, const double *cost, const int *tilem, int grid, int *team, int *bptr,
                                 int *blist, int *queue, int *nqueue)
{
    if (nitems < 0 || grid < 1 || (nitems > 0 && (!cost || !tilem || !team || !queue)) || !bptr || !nqueue ||
        (nitems > 0 && !blist))
        return MF_ERR_INVALID;
    for (int t = 0; t < nitems; t++)
        if (!(cost[t] >= 0.0) || tilem[t] < 0) return MF_ERR_INVALID;
    return mf_batch_schedule_impl(nitems, cost, tilem, grid, team, bptr, blist, queue, nqueue);
}

// Greedy longest-processing-time split of whole systems over nparts GPUs: the
// systems by decreasing cost (ties: lower index first), each to the part with
// the least load so far (ties: lower part).  A system's cost is the sum over its
// work items (groups of <= cap columns) of the queue's item cost.  Host only;
// every rank computes the same split from the same inputs.
extern "C" int mf_batch_partition(int nsys, const int *n, const long long *nnz, const int *nrhs, int cap,
                                  int nparts, int *part, double *load)
{
    if (nsys < 0 || nparts < 1 || (nsys > 0 && (!n || !nnz || !nrhs || !part))) return MF_ERR_INVALID;
    if (cap <= 0) cap = 8;
    if (cap > 8) return MF_ERR_INVALID;
    std::vector<double> cost(nsys, 0.0);
    for (int k = 0; k < nsys; k++) {
        if (n[k] < 1 || nnz[k] < 0 || nrhs[k] < 1) return MF_ERR_INVALID;
        for (int c0 = 0; c0 < nrhs[k]; c0 += cap)
            cost[k] += mf_batch_item_cost(nnz[k], n[k], mf_batch_width(std::min(cap, nrhs[k] - c0)));
    }
    std::vector<int> order(nsys);
    for (int k = 0; k < nsys; k++) order[k] = k;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<double> ld(nparts, 0.0);
    for (int k : order) {
        int best = 0;
        for (int q = 1; q < nparts; q++)
            if (ld[q] < ld[best]) best = q;
        part[k] = best;
        ld[best] += cost[k];
    }
    if (load)
        for (int q = 0; q < nparts; q++) load[q] = ld[q];
    return MF_SUCCESS;
}

extern "C" int mf_spmv(mf_matrix A, const double *x, double *y, int precision, int device_ptrs, void *stream,
                       double *elapsed_ms)
{
    NvtxRange nvtx_range("mf_spmv");
    if (!A || !x || !y) return MF_ERR_INVALID;
    if (precision != MF_PREC_FP64 && precision != MF_PREC_MIXED) return MF_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const double *dxp = x;
    double *dyp = y;
    double *tmp = nullptr;
    if (!device_ptrs) {
        MF_TRY(stage_get(A, ((size_t)A->n_cols + A->n_rows) * sizeof(double) + 16, &tmp));
        MF_CUDA_TRY(cudaMemcpyAsync(tmp, x, (size_t)A->n_cols * sizeof(double), cudaMemcpyHostToDevice, s));
        dxp = tmp;
        dyp = tmp + A->n_cols;
    }
    int rc = mf_spmv_run(A, dxp, dyp, precision, s, elapsed_ms);
    if (!device_ptrs) {
        cudaMemcpyAsync(y, dyp, (size_t)A->n_rows * sizeof(double), cudaMemcpyDeviceToHost, s);
        MF_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return rc;
}

extern "C" int mf_debug_spmv_tiles(mf_matrix A, const double *x, double *y, int tile_prec, int device_ptrs)
{
    if (!A || !x || !y || tile_prec < 0 || tile_prec > 3) return MF_ERR_INVALID;
    const double *dxp = x;
    double *dyp = y, *tmp = nullptr;
    if (!device_ptrs) {
        MF_CUDA_TRY(cudaMalloc((void **)&tmp, ((size_t)A->n_cols + A->n_rows) * sizeof(double) + 16));
        MF_CUDA_TRY(cudaMemcpy(tmp, x, (size_t)A->n_cols * sizeof(double), cudaMemcpyHostToDevice));
        dxp = tmp;
        dyp = tmp + A->n_cols;
    }
    // tile_prec 0..3 are the entry precision codes MF_P64, MF_P32, MF_P16, MF_P8
    int rc = mf_spmv_tiles_run(A, dxp, dyp, tile_prec, 0, nullptr);
    if (!device_ptrs) {
        if (rc == MF_SUCCESS) cudaMemcpy(y, dyp, (size_t)A->n_rows * sizeof(double), cudaMemcpyDeviceToHost);
        cudaFree(tmp);
    }
    return rc;
}

extern "C" int mf_debug_spmm(mf_matrix A, const double *X, double *Y, int tensor_cores, int device_ptrs,
                             double *elapsed_ms)
{
    if (!A || !X || !Y) return MF_ERR_INVALID;
    const size_t nx = (size_t)8 * A->n_cols, ny = (size_t)8 * A->n_rows;
    const double *dX = X;
    double *dY = Y, *tmp = nullptr;
    if (!device_ptrs) {
        MF_TRY(stage_get(A, (nx + ny) * sizeof(double), &tmp));
        MF_CUDA_TRY(cudaMemcpy(tmp, X, nx * sizeof(double), cudaMemcpyHostToDevice));
        dX = tmp;
        dY = tmp + nx;
    }
    int rc = mf_spmm_run(A, dX, dY, tensor_cores ? 1 : 0, 0, elapsed_ms);
    if (!device_ptrs && rc == MF_SUCCESS) MF_CUDA_TRY(cudaMemcpy(Y, dY, ny * sizeof(double), cudaMemcpyDeviceToHost));
    return rc;
}

extern "C" int mf_debug_solver_labels(mf_matrix A, int *vis, int nseg)
{
    if (!A || (nseg > 0 && !vis)) return MF_ERR_INVALID;
    return mf_solver_labels_run(A, vis, nseg);
}

extern "C" int mf_spmv_noalloc(mf_matrix A, const double *x, double *y, int precision, void *stream)
{
    if (!A || !x || !y) return MF_ERR_INVALID;
    if (precision != MF_PREC_FP64 && precision != MF_PREC_MIXED) return MF_ERR_INVALID;
    return mf_spmv_noalloc_run(A, x, y, precision, (cudaStream_t)stream);
}

extern "C" int mf_debug_ref_labels(const double *p_old, const double *p_new, int nseg, int *vis, int device_ptrs)
{
    if (nseg < 0 || (nseg > 0 && (!p_old || !p_new || !vis))) return MF_ERR_INVALID;
    MF_TRY(device_ready());
    if (nseg == 0) return MF_SUCCESS;
    const size_t nv = (size_t)nseg * MF_BS * sizeof(double);
    if (device_ptrs) return mf_ref_labels_run(p_old, p_new, nseg, vis, 0);
    double *d = nullptr;
    int *dv = nullptr;
    MF_CUDA_TRY(cudaMalloc((void **)&d, 2 * nv));
    MF_CUDA_TRY(cudaMalloc((void **)&dv, (size_t)nseg * sizeof(int)));
    cudaMemcpy(d, p_old, nv, cudaMemcpyHostToDevice);
    cudaMemcpy(d + (size_t)nseg * MF_BS, p_new, nv, cudaMemcpyHostToDevice);
    int rc = mf_ref_labels_run(d, d + (size_t)nseg * MF_BS, nseg, dv, 0);
    if (rc == MF_SUCCESS) cudaMemcpy(vis, dv, (size_t)nseg * sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    cudaFree(dv);
    return rc;
}

// ------------------------------------------------------------------ drop-in shims
namespace {

void append_csv(const char *csv, const char *filename, const char *line)
{
    FILE *f = fopen(csv, "a");
    if (!f) return;
    fprintf(f, "%s,%s", filename ? filename : "", line);
    fclose(f);
}

// The full report of the calling thread's last drop-in solve (mf_dropin_last_report).
thread_local mf_report g_dropin_report;

// Shared body of the cg_solve_* shims (main-cg-mixed.cu:2248-3069 / main-cg.cu).
void cg_dropin(int precision, const char *csv, int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x,
               double *b, int n, char *filename, int nnzR, int ori, int max_iter, CgBenchResult *bench_result,
               int skip_output)
{
    const int rowA = (n / MF_BS) * MF_BS;      // main-cg-mixed.cu:2254
    if (x) memset(x, 0, sizeof(double) * (size_t)n);
    mf_matrix A = nullptr;
    int rc = mf_matrix_create(&A, rowA, ori, nnzR, RowPtr, ColIdx, Val, Val_Low, 0, nullptr);
    CgBenchResult res = {0.0, 0, NAN, NAN};
    if (rc == MF_SUCCESS) {
        mf_options o;
        mf_options_default(&o);
        o.precision = precision;
        o.max_iter = max_iter;
        o.fixed_iters = 1;
        o.replace_every = 0;
        mf_report rep;
        memset(&rep, 0, sizeof(rep));
        rc = mf_solve(A, b, x, &o, &rep, 0, nullptr);
        g_dropin_report = rep;
        res.time_ms = rep.time_ms;
        res.iterations = rep.iterations;
        res.l2_norm = rep.relres_true;
        res.residual = rep.residual;
        mf_matrix_destroy(A);
    }
    if (rc != MF_SUCCESS) fprintf(stderr, "millefeuille: %s\n", mf_status_string(rc));
    if (bench_result) *bench_result = res;
    if (!skip_output) {
        printf("time_cg: %f ms\n", res.time_ms);
        char line[256];
        snprintf(line, sizeof(line), "%d,%.3f,%d,%e,%e\n", max_iter, res.time_ms, nnzR, res.l2_norm, res.residual);
        append_csv(csv, filename, line);
    }
}

// Shared body of the bicgstab shims (main-bicg-mixed.cu:1355-2167, main-bicg.cu:13-1335).
int bicg_dropin(int precision, const char *csv, int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x,
                int nnzR, char *filename, int n)
{
    const int colA = n;
    const int rowA = (n / MF_BS) * MF_BS;
    // rhs is overwritten with the row sums A * 1 (main-bicg-mixed.cu:1843-1847)
    for (int i = 0; i < rowA; i++) {
        double sum = 0.0;
        for (int j = RowPtr[i]; j < RowPtr[i + 1]; j++) sum += Val[j];
        rhs[i] = sum;
    }
    if (x) memset(x, 0, sizeof(double) * (size_t)rowA);
    mf_matrix A = nullptr;
    int rc = mf_matrix_create(&A, rowA, colA, nnzR, RowPtr, ColIdx, Val, nullptr, 0, nullptr);
    mf_report rep;
    memset(&rep, 0, sizeof(rep));
    if (rc == MF_SUCCESS) {
        mf_options o;
        mf_options_default(&o);
        o.method = MF_METHOD_BICGSTAB;
        o.precision = precision;
        o.max_iter = 50;          // fixed 50 iterations (main-bicg-mixed.cu:224)
        o.fixed_iters = 1;
        o.replace_every = 0;
        rc = mf_solve(A, rhs, x, &o, &rep, 0, nullptr);
        mf_matrix_destroy(A);
    }
    g_dropin_report = rep;
    if (rc != MF_SUCCESS) fprintf(stderr, "millefeuille: %s\n", mf_status_string(rc));
    printf("time_bicg=%lf ms\n", rep.time_ms);
    char line[256];
    snprintf(line, sizeof(line), "%d,%.3f,%d,%e,%e\n", 50, rep.time_ms, nnzR, rep.relres_true,
             rep.relres_true);
    append_csv(csv, filename, line);
    return rc == MF_SUCCESS ? 0 : 1;
}

}  // namespace

// The reference has two cg_solve_inc with one signature: the mixed-precision
// solver of main-cg-mixed.cu:2248 and the FP64 one of main-cg.cu:1110 (which
// main-cg calls for nnz < 10,000, main-cg.cu:1727-1745).  libmillefeuille.so
// exports the mixed one; libmillefeuille_fp64.so, the same objects with this
// file compiled with MF_CG_INC_FP64, exports the FP64 one, for programs that
// link main-cg.cu's entry points.
extern "C" void cg_solve_inc(int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x, double *b, int n,
                             int *iter, int maxiter, double threshold, char *filename, int nnzR, int ori,
                             int max_iter, CgBenchResult *bench_result, int skip_output)
{
    (void)iter; (void)maxiter; (void)threshold;
#ifdef MF_CG_INC_FP64
    cg_dropin(MF_PREC_FP64, "cg_performance.csv", RowPtr, ColIdx, Val, Val_Low, x, b, n, filename, nnzR, ori,
              max_iter, bench_result, skip_output);
#else
    cg_dropin(MF_PREC_MIXED, "cg_mixed_performance.csv", RowPtr, ColIdx, Val, Val_Low, x, b, n, filename, nnzR,
              ori, max_iter, bench_result, skip_output);
#endif
}

extern "C" int mf_dropin_last_report(mf_report *out)
{
    if (!out) return MF_ERR_INVALID;
    *out = g_dropin_report;
    return MF_SUCCESS;
}

extern "C" void cg_solve_sync(int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x, double *b, int n,
                              int *iter, int maxiter, double threshold, char *filename, int nnzR, int ori,
                              int max_iter, CgBenchResult *bench_result, int skip_output)
{
    (void)iter; (void)maxiter; (void)threshold;
    cg_dropin(MF_PREC_FP64, "cg_performance.csv", RowPtr, ColIdx, Val, Val_Low, x, b, n, filename, nnzR, ori,
              max_iter, bench_result, skip_output);
}

extern "C" void cg_solve_reduce(int *RowPtr, int *ColIdx, double *Val, float *Val_Low, double *x, double *b,
                                int n, int *iter, int maxiter, double threshold, char *filename, int nnzR, int ori,
                                int max_iter, CgBenchResult *bench_result, int skip_output)
{
    (void)iter; (void)maxiter; (void)threshold;
    cg_dropin(MF_PREC_FP64, "cg_performance.csv", RowPtr, ColIdx, Val, Val_Low, x, b, n, filename, nnzR, ori,
              max_iter, bench_result, skip_output);
}

extern "C" int bicgstab(int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x, int nnzR, char *filename,
                        int n)
{
    return bicg_dropin(MF_PREC_MIXED, "bicg_mixed_performance.csv", RowPtr, ColIdx, Val, rhs, x, nnzR, filename,
                       n);
}

extern "C" int bicgstab_sync(int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x, int nnzR,
                             char *filename, int n)
{
    return bicg_dropin(MF_PREC_FP64, "bicg_performance.csv", RowPtr, ColIdx, Val, rhs, x, nnzR, filename, n);
}

extern "C" int bicgstab_inc(int *RowPtr, int *ColIdx, double *Val, double *rhs, double *x, int nnzR,
                            char *filename, int n)
{
    return bicg_dropin(MF_PREC_FP64, "bicg_performance.csv", RowPtr, ColIdx, Val, rhs, x, nnzR, filename, n);
}
