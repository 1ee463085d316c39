// solver.cu -- the persistent single-kernel CG / BiCGSTAB and the tile SpMV.
//
// One cooperative launch runs the whole solve (the reference's single-kernel
// design, Mille-feuille-cg.h:1113-1348 / main-cg-mixed.cu:1016-1385 /
// main-bicg-mixed.cu:122-723), re-designed for sm_100a:
//  * grid = SMs x resident blocks (cooperative launch guarantees co-residency);
//  * a half-warp owns a contiguous range of tile-rows (lane i = row 16R+i) for
//    every phase, so y rows are written by their owner only (no y atomics) and
//    every dot product is reduced in a fixed order (deterministic);
//  * the tile SpMV walks the half-warp's solver slices: one 16-byte header per
//    slice, the slice's tile words held one tile per lane (read with
//    __shfl_sync), the next slice's descriptor loaded while the current slice's
//    value + x loads are in flight;
//  * the grid barrier is a monotone counter: fence + relaxed arrive, relaxed
//    polls, one acquire fence, every wait bounded by %globaltimer (MF_ERR_TIMEOUT);
//  * dot products: warp shuffle tree -> per-block partial in a fixed slot ->
//    after the barrier each block sums the partials in the same order;
//  * matrix payload is streamed with evict-first loads so the vectors stay in L2.
#include "mf_internal.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kRedKinds = 10;     // reduction slot groups
constexpr int kRedWidth = 4;      // doubles per group per block
constexpr int kDefaultLB = 2;     // default register-budget variant of the persistent kernel
constexpr int kVB = 4;            // tile-rows per step in the vector phases (loads in flight)
constexpr int kDemoteCool = 16;   // SpMVs without per-slice lookups after one that did not pay

enum { MODE_FP64 = 0, MODE_MIXED = 1, MODE_PARITY = 2 };

// ------------------------------------------------------------ bounds checks
// The bounds-checked build (-DMF_CHECK, libmillefeuille_check.so): every index
// the kernels take from stored data -- a half-warp's slice range, a tile word's
// column tile, a per-tile table entry, a slice's payload, a gathered vector
// position, an epilogue tile-row, a batch queue entry -- is compared with the
// extent of the array it addresses before the access.  A failed check keeps the
// first (site, index, limit) of the device in g_chk and the access is skipped
// (a load reads zero, a store or a slice is dropped); the entry point that
// launched the kernel returns MF_ERR_CHECK.  Nothing traps: the context stays
// usable.  In the normal build chk_in() is `true` and the checks compile away.
enum { CHK_SLICE = 1, CHK_TILE, CHK_PAYLOAD, CHK_X, CHK_ROWLEN, CHK_ROW, CHK_ITEM, CHK_NSITES };
#ifdef MF_CHECK
__device__ unsigned long long g_chk[3];   // site, index, limit of the first failed check

__device__ __noinline__ void chk_fail(int site, long long idx, long long lim)
{
    if (atomicCAS(&g_chk[0], 0ull, (unsigned long long)site) == 0ull) {
        g_chk[1] = (unsigned long long)idx;
        g_chk[2] = (unsigned long long)lim;
    }
}

__device__ __forceinline__ bool chk_in(int site, long long idx, long long lim)
{
    if (idx >= 0 && idx < lim) return true;
    chk_fail(site, idx, lim);
    return false;
}
#else
__device__ __forceinline__ bool chk_in(int, long long, long long) { return true; }
#endif

struct SolverParams {
    int n, tilem, vec_len;
    const int *rowptr;            // CSR row pointers (entry counts of the lean FP32 walk)
    const int *seg_ptr;
    const int4 *seg_hdr;
    const uint16_t *seg_rowlen;
    const unsigned char *meta;
    const double *v64;
    const float *v32;
    const __half *v16;
    const int8_t *v8, *v8ref;
    const int *tile_col;
    const int *seg_tile;          // [nseg*16] tile words: column-tile << 8 | caps
    const int *tile_off;          // csr_offset: tile payload offsets (tile nnz for the counters)
    const float *i8_scale;
    const unsigned char *tile_caps;
    const int *hw_begin;
    const double *b;
    double *x, *r, *p, *q, *rh, *s, *t;
    float *p32, *s32, *mag_p, *mag_s;
    float *mag_r;                 // CG with the SpMV on r: r's segment magnitudes
    __half *p16, *s16;
    int8_t *p8, *s8;
    signed char *lab_p, *lab_s;
    double *red;
    unsigned int *bar;
    int *err;
    double *out;
    unsigned long long *counts;
    unsigned long long *phase_ns;   // [8] block-0 time per phase: spmv, vecB, vecC, barrier, replacement
    int method, max_iter, fixed_iters, replace_every, use_lossless;
    int x0_given;                 // x holds the initial guess: r = b - A x at the start
    int lossless_any;             // use_lossless and enough tiles are exact in INT8 / FP16
    float min_demoted;            // mixed: a dynamic SpMV that runs fewer tiles than this below FP32
                                  // turns the operand's per-slice lookups off for kDemoteCool SpMVs
    float min_small;              // mixed: narrower tiles only when at least this many column
                                  // segments were small in the operand's previous update
    double tol;
    float demote16, demote8;
    unsigned long long timeout_ns;
    int stall_first_barrier;   // test hook: first barrier expects one extra arrival
    float relax_eta;           // mixed CG: relaxation factor of the matvec precision (0: off)
    int relax_int8;            // the relaxation may go down to scaled INT8 (else FP16 at most)
    int fp16_ok;               // every tile's values are within FP16's normal range
    int lean_f16;              // mixed, use_lossless: every tile is exact in FP16, so the lookup-free
                               // walk runs FP16 stored values (the lossless choice made once)
    // extents for the bounds-checked build: slices, tiles, payload entries, and
    // the operand length its gathers are checked against (vec_len, or less
    // through the test_check_limit hook)
    int nseg, ntiles, chk_xlen;
    long long n_payload;
};

struct Shared {
    double wred[kWarps][kRedWidth];
    double bcast[kRedWidth];
    int flag;
    unsigned cnt[kWarps * 2][10];   // per-half-warp tile / entry counters per precision (mixed / parity)
    unsigned long long clk_t, clk_acc[5];   // block 0 phase clock
};

// ------------------------------------------------------------ grid barrier
template <class SH>
__device__ bool grid_barrier(const SolverParams &P, unsigned &epoch, SH &sh)
{
    __syncthreads();
    epoch += 1;
    if (threadIdx.x == 0) {
        const unsigned long long tw0 = mf_globaltimer();
        const unsigned target = epoch * gridDim.x + ((P.stall_first_barrier && epoch == 1) ? 1u : 0u);
        // fence-release pattern: the block's writes (ordered before by bar.sync) are
        // visible at gpu scope before the arrival; polls are relaxed loads and one
        // acquire fence follows (an acquire load per poll costs like a fence)
        __threadfence();
        mf_red_relaxed_add_u32(P.bar, 1u);
        bool ok = true;
        const unsigned long long t0 = mf_globaltimer();
        unsigned spins = 0;
        for (;;) {
            unsigned v = mf_ld_relaxed_u32(P.bar);
            if ((int)(v - target) >= 0) break;
            if (*(volatile int *)P.err) { ok = false; break; }
            if ((++spins & 63u) == 0u && mf_globaltimer() - t0 > P.timeout_ns) {
                atomicCAS(P.err, 0, MF_ERR_TIMEOUT);
                ok = false;
                break;
            }
        }
        mf_fence_acq_rel_gpu();
        sh.flag = ok ? 1 : 0;
        if (blockIdx.x == 0 && P.phase_ns) P.phase_ns[5] += mf_globaltimer() - tw0;   // block 0 spin time
    }
    __syncthreads();
    return sh.flag != 0;
}

// Block partial of up to 4 sums (mask bit k set -> max instead of sum) written
// to red[kind][k][block] (value-major, so a collect reads consecutive blocks).
__device__ void block_partial(const SolverParams &P, Shared &sh, int kind, double v0, double v1, double v2,
                              double v3, int nv, unsigned maxmask)
{
    double v[kRedWidth] = {v0, v1, v2, v3};
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < kRedWidth; k++) {
        if (k >= nv) break;
        double a = v[k];
        const bool mx = (maxmask >> k) & 1u;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            double b = __shfl_xor_sync(0xffffffffu, a, o);
            a = mx ? fmax(a, b) : a + b;
        }
        if (lane == 0) sh.wred[wib][k] = a;
    }
    __syncthreads();
    if (wib == 0) {
        for (int k = 0; k < nv; k++) {
            const bool mx = (maxmask >> k) & 1u;
            double a = (lane < kWarps) ? sh.wred[lane][k] : (mx ? -1.0e300 : 0.0);
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                double b = __shfl_xor_sync(0xffffffffu, a, o);
                a = mx ? fmax(a, b) : a + b;
            }
            if (lane == 0) P.red[((long long)kind * kRedWidth + k) * gridDim.x + blockIdx.x] = a;
        }
    }
}

// After the barrier: every block sums the partials of `kind` in the same order
// (lane c takes blocks c, c + 32, ... in turn, then a shuffle tree).  Partials
// sit value-major (red[kind][k][block]), warp k reduces value k, and each lane
// issues all its loads before the first add, so the collect costs one L2 round
// trip instead of one per partial.  No trailing barrier: the next writer of
// sh.bcast is the next collect, which every thread reaches only through the
// barriers of block_partial and grid_barrier, after it has read bcast here.
__device__ void grid_collect(const SolverParams &P, Shared &sh, int kind, int nv, unsigned maxmask,
                             double *outv)
{
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    if (wib < nv) {
        const bool mx = (maxmask >> wib) & 1u;
        const double id = mx ? -1.0e300 : 0.0;
        const int G = (int)gridDim.x;
        const double *src = P.red + ((long long)kind * kRedWidth + wib) * G;
        constexpr int kU = 10;              // 320 blocks per pass: the grid of 148 SMs x 2 in one
        double a = id;
        for (int c0 = 0; c0 < G; c0 += 32 * kU) {
            double t[kU];
#pragma unroll
            for (int j = 0; j < kU; j++) {
                const int cb = c0 + lane + 32 * j;
                t[j] = cb < G ? src[cb] : id;
            }
#pragma unroll
            for (int j = 0; j < kU; j++) a = mx ? fmax(a, t[j]) : a + t[j];
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const double b = __shfl_xor_sync(0xffffffffu, a, o);
            a = mx ? fmax(a, b) : a + b;
        }
        if (lane == 0) sh.bcast[wib] = a;
    }
    __syncthreads();
    for (int k = 0; k < nv; k++) outv[k] = sh.bcast[k];
}

// ------------------------------------------------------------ tile SpMV
// Reference-rule label code (d_vis) -> entry precision.
__device__ __forceinline__ int parity_prec(int code)
{
    return code == 0 ? MF_P64 : code == 4 ? MF_P32 : code == 3 ? MF_P16 : code == 2 ? MF_P8 : MF_PSKIP;
}

// The x operands of one SpMV: the FP64 vector (FP64 and mixed modes multiply
// every stored precision against it), and in parity mode its FP32 / FP16 /
// INT8 shadows; mag / lab are the per-column-segment statistics the precision
// choice reads.
struct XVec {
    const double *x64;
    const float *x32;
    const __half *x16;
    const int8_t *x8;
    const float *mag;
    const signed char *lab;
    float invM;
    int force_pr;            // >= 0: every tile in this precision
    int dyn;                 // mixed: 0 = no tile can leave the base precision (no precision lookups)
    int lean_pr;             // mixed: the base precision of the lookup-free walk (FP32, or FP16 when
                             // every tile is exact in FP16)
};

// Tile table of a slice, one tile per lane (lane i holds slot i).
struct TileReg {
    int xb;       // column-tile * 16
    int pr;       // entry precision of the tile (the slice runs at the half's minimum)
};

__device__ __forceinline__ int hdr_kp(int4 h) { return h.z & 0xFFFF; }
__device__ __forceinline__ int hdr_nt(int4 h) { return (h.z >> 16) & 0xFF; }
__device__ __forceinline__ bool hdr_last(int4 h) { return (h.z >> 24) & 1; }
__device__ __forceinline__ long long hdr_off(int4 h) { return (long long)h.w << 7; }

// The precision statistic of lane i's tile (tile word tw = column-tile << 8 |
// caps): the column segment's magnitude (mixed mode) or its reference label
// (parity mode).  Issued one slice ahead so its latency overlaps a slice.
template <int MODE, bool F64>
__device__ __forceinline__ float load_stat(const XVec &X, int tw, int i, int nt)
{
    if (F64 || MODE == MODE_FP64 || i >= nt || X.force_pr >= 0 || (MODE == MODE_MIXED && !X.dyn)) return 0.0f;
    const int jc = tw >> 8;
    if (MODE == MODE_MIXED) return X.mag[jc];
    return (float)X.lab[jc];
}

// Entry precision of lane i's tile from its tile word and statistic.
template <int MODE, bool F64>
__device__ __forceinline__ int tile_prec(const SolverParams &P, int tw, float st, const XVec &X)
{
    if (F64 || MODE == MODE_FP64) return MF_P64;
    if (X.force_pr >= 0) return X.force_pr;
    if (MODE == MODE_PARITY) return parity_prec((int)st);
    if (!X.dyn) return MF_P32;
    const unsigned cap = (unsigned)tw & 0xFFu;
    const float rel = st * X.invM;
    int pr = MF_P32;
    if (rel <= P.demote8) pr = MF_P8;
    else if (rel <= P.demote16 && (cap & MF_CAP_FP16_OK)) pr = MF_P16;
    if (P.use_lossless) {
        if (cap & MF_CAP_EXACT_I8) pr = MF_P8;
        else if ((cap & MF_CAP_EXACT_F16) && pr == MF_P32) pr = MF_P16;
    }
    return pr;
}

// Lane i's 8 stored values of the chunk whose payload starts at entry cb (a
// multiple of 128), in precision PR: 128-bit loads of the row's 16-byte groups
// (4 for FP64, 2 for FP32, 1 for FP16; an 8-byte load for INT8), each issued
// only when its first entry lies inside the row (nact entries of the row fall
// in this chunk; the stored padding past a row's end is zero).  FP32 / FP16 /
// INT8 values come back as float (INT8 unscaled).
template <int PR>
__device__ __forceinline__ void load_chunk(const SolverParams &P, long long cb, int i, int nact,
                                           double (&v64)[8], float (&v)[8])
{
    if (PR == MF_P64) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            double2 d = make_double2(0.0, 0.0);
            if (2 * q < nact) d = __ldcs((const double2 *)(P.v64 + cb + 32 * q) + i);
            v64[2 * q] = d.x;
            v64[2 * q + 1] = d.y;
        }
    } else if (PR == MF_P32) {
#pragma unroll
        for (int q = 0; q < 2; q++) {
            float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
            if (4 * q < nact) f = __ldcs((const float4 *)(P.v32 + cb + 64 * q) + i);
            v[4 * q] = f.x;
            v[4 * q + 1] = f.y;
            v[4 * q + 2] = f.z;
            v[4 * q + 3] = f.w;
        }
    } else if (PR == MF_P16) {
        uint4 u = make_uint4(0u, 0u, 0u, 0u);
        if (nact > 0) u = __ldcs((const uint4 *)(P.v16 + cb) + i);
        const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int q = 0; q < 4; q++) {
            v[2 * q] = __half2float(__ushort_as_half((unsigned short)(w[q] & 0xFFFFu)));
            v[2 * q + 1] = __half2float(__ushort_as_half((unsigned short)(w[q] >> 16)));
        }
    } else {
        uint2 u = make_uint2(0u, 0u);
        if (nact > 0) u = __ldcs((const uint2 *)(P.v8 + cb) + i);
#pragma unroll
        for (int j = 0; j < 8; j++) v[j] = (float)(int8_t)(((j < 4 ? u.x : u.y) >> (8 * (j & 3))) & 0xFFu);
    }
}

// Uniform-precision chunk loop: every entry of the slice is stored in
// precision PR (FP64, FP32, FP16 or scaled INT8); the value is widened to FP64
// in registers and multiplied with the FP64 x, so the row sum is FP64 and only
// the stored values are rounded.  The kernel waits on memory, not on the FP64
// pipe: against FP32 products with an FP32 copy of x this measured 6 % fewer
// iterations on the 128^3 variable-coefficient system at the same time per
// iteration, and needs no FP32 copy of the operand.
// A slice is kp/8 chunks of 16 rows x 8 entries.  Per chunk the value loads
// are issued first (they need only the slice offset, known at the top of the
// slice), then the index word, then the gathered x; pre() issues the next
// slice's dependent loads once the first chunk is in flight.
// No row lengths: a row's padding entries are stored as value 0 with index
// byte 0 (slot 0, column 0), so a lane loads and gathers all kp entries of its
// row and the padding adds 0 * x.  Against loads and gathers predicated on
// per-lane row-length words this measured 15 % faster on the 128^3 FP64 solve.
template <int PR, typename Pre>
__device__ __forceinline__ double slice_dot_uniform(const SolverParams &P, int4 h, long long off, int i,
                                                    unsigned hmask, const TileReg &T, const XVec &X, Pre &pre)
{
    const int kp = hdr_kp(h);
    float sc = 0.0f;
    if (PR == MF_P8) sc = (i < hdr_nt(h) && chk_in(CHK_TILE, h.x + i, P.ntiles)) ? P.i8_scale[h.x + i] : 0.0f;
    // (uniform over the half-warp: the slice is skipped by all 16 lanes)
    if (!chk_in(CHK_PAYLOAD, off + (long long)kp * MF_BS - 1, P.n_payload)) return 0.0;
    double acc = 0.0;
    for (int k0 = 0; k0 < kp; k0 += 8) {
        const long long cb = off + (long long)(k0 >> 3) * 128;
        double v64[8];
        float v[8];
        load_chunk<PR>(P, cb, i, 8, v64, v);
        const unsigned long long m8 = __ldcs((const unsigned long long *)(P.meta + cb) + i);
        double xv[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const unsigned mm = (unsigned)(m8 >> (8 * j)) & 0xFFu;
            const int slot = (int)(mm >> 4);
            const int xi = __shfl_sync(hmask, T.xb, slot, 16) + (int)(mm & 15u);
            xv[j] = chk_in(CHK_X, xi, P.chk_xlen) ? X.x64[xi] : 0.0;
            if (PR == MF_P8) v[j] *= __shfl_sync(hmask, sc, slot, 16);
        }
        if (k0 == 0) pre();
#pragma unroll
        for (int j = 0; j < 8; j++) acc = fma(PR == MF_P64 ? v64[j] : (double)v[j], xv[j], acc);
    }
    return acc;
}

// Row i of one slice times x.  The 8 entries of a chunk are loaded together
// (value + gathered x), then accumulated; occupancy (32 warps per SM at 64
// registers) hides part of the memory latency.  Variants with more loads in
// flight per thread (two chunks, or 3-4 blocks per SM at 32-42 registers)
// spilled and were slower.  In mixed mode a slice runs in one precision, the
// most conservative of its tiles' labels (no per-entry dispatch).
template <int MODE, bool F64, typename Pre>
__device__ __forceinline__ double slice_dot(const SolverParams &P, int4 h, int i, unsigned hmask, long long off,
                                            const TileReg &T, const XVec &X, unsigned *cnt, Pre &pre)
{
    // precision codes order FP64 < FP32 < FP16 < INT8: the minimum is the most precise
    int pr = MF_P64;
    if (!(MODE == MODE_FP64 || F64)) {
        pr = __reduce_min_sync(hmask, (i < hdr_nt(h)) ? T.pr : MF_P8);
    }
    if (cnt && i == 0 && chk_in(CHK_TILE, (long long)h.x + hdr_nt(h), (long long)P.ntiles + 1)) {
        // the half-warp's own counter slots (lane 0 writes, no atomics): tile
        // products and entries of the executed precision (the slice's tiles
        // are consecutive, so its entries are a difference of tile payload
        // offsets); a half-warp's counts stay far below 2^32 per solve
        cnt[pr] += (unsigned)hdr_nt(h);
        cnt[5 + pr] += (unsigned)(P.tile_off[h.x + hdr_nt(h)] - P.tile_off[h.x]);
    }
    if (MODE == MODE_FP64 || F64) return slice_dot_uniform<MF_P64>(P, h, off, i, hmask, T, X, pre);
    if (pr == MF_P32) return slice_dot_uniform<MF_P32>(P, h, off, i, hmask, T, X, pre);
    if (pr == MF_P64) return slice_dot_uniform<MF_P64>(P, h, off, i, hmask, T, X, pre);
    if (pr == MF_P16) return slice_dot_uniform<MF_P16>(P, h, off, i, hmask, T, X, pre);
    return slice_dot_uniform<MF_P8>(P, h, off, i, hmask, T, X, pre);
}

// Parity mode: the reference's tile arithmetic (main-cg-mixed.cu:1130-1214):
// per (tile,row) two partial sums (even / odd entry positions, the lane pair of
// the reference), each in the tile's precision -- FP64 fma, FP32 fmaf, FP16
// __hfma on half x, INT8 in int8 on truncated x -- bypass tiles skipped; the
// partials are added to the FP64 row sum, even then odd.
__device__ __forceinline__ void parity_flush(double &acc, int pr, const double *a64, const float *a32,
                                             const __half *a16, const int8_t *a8)
{
    for (int q = 0; q < 2; q++) {
        if (pr == MF_P64) acc += a64[q];
        else if (pr == MF_P32) acc += (double)a32[q];
        else if (pr == MF_P16) acc += (double)__half2float(a16[q]);
        else if (pr == MF_P8) acc += (double)a8[q];
    }
}

__device__ __forceinline__ double slice_dot_parity(const SolverParams &P, int4 h, int i, unsigned hmask, int len,
                                                   const TileReg &T, const XVec &X)
{
    const int kp = hdr_kp(h);
    const long long off = hdr_off(h);
    if (!chk_in(CHK_PAYLOAD, off + (long long)kp * MF_BS - 1, P.n_payload)) return 0.0;
    double acc = 0.0;
    double a64[2] = {0.0, 0.0};
    float a32[2] = {0.0f, 0.0f};
    __half a16[2] = {__float2half_rn(0.0f), __float2half_rn(0.0f)};
    int8_t a8[2] = {0, 0};
    int cur_slot = -1, cur_pr = MF_PSKIP, pos = 0;
    for (int k = 0; k < kp; k++) {
        const bool act = k < len;
        const unsigned mm = act ? (unsigned)P.meta[mf_slot<1>(off, k, i)] : 0u;
        const int slot = (int)(mm >> 4);
        const int xi = __shfl_sync(hmask, T.xb, slot, 16) + (int)(mm & 15u);
        const int pr = __shfl_sync(hmask, T.pr, slot, 16);
        if (!act || !chk_in(CHK_X, xi, P.chk_xlen)) continue;
        if (slot != cur_slot) {
            parity_flush(acc, cur_pr, a64, a32, a16, a8);
            a64[0] = a64[1] = 0.0;
            a32[0] = a32[1] = 0.0f;
            a16[0] = a16[1] = __float2half_rn(0.0f);
            a8[0] = a8[1] = 0;
            cur_slot = slot;
            cur_pr = pr;
            pos = 0;
        }
        const int q = pos & 1;
        if (pr == MF_P64) a64[q] = fma(X.x64[xi], P.v64[mf_slot<8>(off, k, i)], a64[q]);
        else if (pr == MF_P32) a32[q] = fmaf(X.x32[xi], P.v32[mf_slot<4>(off, k, i)], a32[q]);
        else if (pr == MF_P16) a16[q] = __hfma(X.x16[xi], P.v16[mf_slot<2>(off, k, i)], a16[q]);
        else if (pr == MF_P8) a8[q] = (int8_t)((int)a8[q] + (int)X.x8[xi] * (int)P.v8ref[mf_slot<1>(off, k, i)]);
        pos++;
    }
    parity_flush(acc, cur_pr, a64, a32, a16, a8);
    return acc;
}

// Lane i's tile word and row length of slice s (header h).  The bounds-checked
// build checks the tile word's column tile against the operand length and the
// row length against the slice width; a word that fails reads as 0 (column
// tile 0, an empty row).
__device__ __forceinline__ int load_tw(const SolverParams &P, int s, int i)
{
    const int tw = P.seg_tile[(long long)s * MF_BS + i];
    return chk_in(CHK_TILE, (long long)(tw >> 8) * MF_BS, P.chk_xlen) ? tw : 0;
}

__device__ __forceinline__ int load_len(const SolverParams &P, int s, int i, int4 h)
{
    const int len = P.seg_rowlen[(long long)s * MF_BS + i];
    return chk_in(CHK_ROWLEN, len, hdr_kp(h) + 1) ? len : 0;
}

// One chunk of the lean walk: lane i's 8 stored values of a uniform-precision
// slice (FP64: four 16-byte loads; FP32: two; FP16: one) and its index word,
// loaded unpredicated (the stored padding past a row's end is zero).
template <int PR> struct LeanChunk;

template <> struct LeanChunk<MF_P64> {
    double2 d[4];
    unsigned long long m;
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int q = 0; q < 4; q++) d[q] = make_double2(0.0, 0.0);
        m = 0ull;
    }
    __device__ __forceinline__ void load(const SolverParams &P, long long cb, int i)
    {
#pragma unroll
        for (int q = 0; q < 4; q++) d[q] = __ldcs((const double2 *)(P.v64 + cb + 32 * q) + i);
        m = __ldcs((const unsigned long long *)(P.meta + cb) + i);
    }
    __device__ __forceinline__ void values(double (&v)[8]) const
    {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            v[2 * q] = d[q].x;
            v[2 * q + 1] = d[q].y;
        }
    }
};

template <> struct LeanChunk<MF_P32> {
    float4 a, b;
    unsigned long long m;
    __device__ __forceinline__ void zero()
    {
        a = b = make_float4(0.f, 0.f, 0.f, 0.f);
        m = 0ull;
    }
    __device__ __forceinline__ void load(const SolverParams &P, long long cb, int i)
    {
        a = __ldcs((const float4 *)(P.v32 + cb) + i);
        b = __ldcs((const float4 *)(P.v32 + cb + 64) + i);
        m = __ldcs((const unsigned long long *)(P.meta + cb) + i);
    }
    __device__ __forceinline__ void values(double (&v)[8]) const
    {
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
        v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    }
};

template <> struct LeanChunk<MF_P16> {
    uint4 u;
    unsigned long long m;
    __device__ __forceinline__ void zero()
    {
        u = make_uint4(0u, 0u, 0u, 0u);
        m = 0ull;
    }
    __device__ __forceinline__ void load(const SolverParams &P, long long cb, int i)
    {
        u = __ldcs((const uint4 *)(P.v16 + cb) + i);
        m = __ldcs((const unsigned long long *)(P.meta + cb) + i);
    }
    __device__ __forceinline__ void values(double (&v)[8]) const
    {
        const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int q = 0; q < 4; q++) {
            v[2 * q] = (double)__half2float(__ushort_as_half((unsigned short)(w[q] & 0xFFFFu)));
            v[2 * q + 1] = (double)__half2float(__ushort_as_half((unsigned short)(w[q] >> 16)));
        }
    }
};

// The lean walk: every slice of the range runs stored precision PR (the FP64
// mode; mixed mode when no tile can leave the base precision in this SpMV --
// FP32, or FP16 when every tile is exact in FP16; the standalone SpMVs), no
// per-slice precision reduction; the range's tile and entry totals go to the
// counters once, at the end (entries from the CSR row pointers of the range's
// tile-rows).
// The walk reads no row lengths: a row's padding entries are stored as value
// 0 with index byte 0 (slot 0, column 0), so for them a lane gathers x at the
// slice's first tile column and adds 0 * x.  Without the per-lane row-length
// words (and their predicates) the 128^3 mixed solve measured 10 % faster.
// The walk is software-pipelined by one chunk.  A half-warp's slices are
// stored back to back, so its chunks (kp / 8 per slice) form one contiguous
// stream and chunk c + 1 starts 128 entries after chunk c whatever slice it
// belongs to: its values and index word are requested as soon as chunk c's x
// gathers are issued, so their DRAM trip overlaps chunk c's gathers, sum and
// tile-row epilogue instead of following them.  Sums are formed in the same
// order as slice_dot_uniform (per slice from 0, added to the tile-row's sum).
template <int PR, typename Epi>
__device__ __forceinline__ void spmv_range_lean(const SolverParams &P, int sb, int se, int i, unsigned hmask,
                                                const XVec &X, unsigned *cnt, Epi &epi)
{
    int4 h = P.seg_hdr[sb];
    const int4 hl = P.seg_hdr[se - 1];
    const long long off0 = hdr_off(h);
    const int nch = (int)((hdr_off(hl) + (long long)hdr_kp(hl) * MF_BS - off0) >> 7);
    if (!chk_in(CHK_PAYLOAD, off0, P.n_payload) || !chk_in(CHK_PAYLOAD, off0 + (long long)nch * 128 - 1, P.n_payload))
        return;
    const int R0 = h.y;
    int tw = load_tw(P, sb, i);
    LeanChunk<PR> cur;
    cur.load(P, off0, i);
    int4 hn = make_int4(0, 0, 0, 0);
    int twn = 0;
    int s = sb, kc = 0, kchunks = hdr_kp(h) >> 3;
    unsigned ntiles = 0;
    double acc = 0.0, sacc = 0.0;
    for (int c = 0; c < nch; c++) {
        if (kc == 0 && s + 1 < se) {       // the next slice's words, one slice ahead
            hn = P.seg_hdr[s + 1];
            twn = load_tw(P, s + 1, i);
        }
        const int xb = (tw >> 8) * MF_BS;
        double xv[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const unsigned mm = (unsigned)(cur.m >> (8 * j)) & 0xFFu;
            const int xi = __shfl_sync(hmask, xb, (int)(mm >> 4), 16) + (int)(mm & 15u);
            xv[j] = chk_in(CHK_X, xi, P.chk_xlen) ? X.x64[xi] : 0.0;
        }
        LeanChunk<PR> nxt;
        nxt.zero();
        if (c + 1 < nch) nxt.load(P, off0 + (long long)(c + 1) * 128, i);
        double v[8];
        cur.values(v);
#pragma unroll
        for (int j = 0; j < 8; j++) sacc = fma(v[j], xv[j], sacc);
        if (++kc == kchunks) {             // the slice is done
            ntiles += (unsigned)hdr_nt(h);
            acc += sacc;
            sacc = 0.0;
            if (hdr_last(h)) {
                if (chk_in(CHK_ROW, h.y, P.tilem)) epi(h.y, acc);
                acc = 0.0;
            }
            s++;
            h = hn;
            tw = twn;
            kc = 0;
            kchunks = hdr_kp(h) >> 3;
        }
        cur = nxt;
    }
    if (cnt && i == 0 && chk_in(CHK_ROW, R0, P.tilem) && chk_in(CHK_ROW, hl.y, P.tilem)) {
        cnt[PR] += ntiles;
        cnt[5 + PR] += (unsigned)(P.rowptr[min(P.n, (hl.y + 1) * MF_BS)] - P.rowptr[R0 * MF_BS]);
    }
}

// y = A x over the half-warp's slices [sb, se); epi(R, y) is called once per
// tile-row (after its last slice) with the row sum of lane i.
// F64: every tile in FP64 (the FP64 residual replacement and the FP64 SpMV).
//
// Descriptor pipeline: a half-warp's slices are stored back to back, so slice
// s+1 starts where slice s ends (offset + 16 * kp).  The words indexed by the
// slice number alone (header, lane i's tile word, and in parity mode its row
// length) are loaded one slice ahead, at the top of the previous slice,
// together with that slice's own loads; the precision statistic (mixed /
// parity) is loaded one slice ahead once the tile word is in.  A slice then
// waits for two round trips: values + index word, then the gathered x.
template <int MODE, bool F64, typename Epi>
__device__ __forceinline__ void spmv_range(const SolverParams &P, int sb, int se, int i, unsigned hmask,
                                           const XVec &X, unsigned *cnt, Epi epi)
{
    if (sb >= se) return;
    if (!chk_in(CHK_SLICE, sb, P.nseg) || !chk_in(CHK_SLICE, se - 1, P.nseg)) return;
    // the FP64 mode takes the pipelined walk too (128^3 FP64 CG 62.0 -> 60.3 ms);
    // the mixed mode's FP64 replacement SpMVs do not: in that kernel the extra
    // code cost the mixed solve more (61.3 -> 62.0 ms) than it saved
    if (MODE == MODE_FP64) {
        spmv_range_lean<MF_P64>(P, sb, se, i, hmask, X, cnt, epi);
        return;
    }
    if (MODE == MODE_MIXED && !F64) {
        const int lean = (X.force_pr < 0 && !X.dyn) ? X.lean_pr : X.force_pr;
        if (lean == MF_P32) {
            spmv_range_lean<MF_P32>(P, sb, se, i, hmask, X, cnt, epi);
            return;
        }
        if (lean == MF_P16) {
            spmv_range_lean<MF_P16>(P, sb, se, i, hmask, X, cnt, epi);
            return;
        }
    }
    // row lengths: parity mode only (its tile arithmetic walks real entries)
    constexpr bool kLen = (MODE == MODE_PARITY && !F64);
    int4 h = P.seg_hdr[sb];
    int tw = load_tw(P, sb, i);
    int len = kLen ? load_len(P, sb, i, h) : 0;
    float st = load_stat<MODE, F64>(X, tw, i, hdr_nt(h));
    long long off = hdr_off(h);
    double acc = 0.0;
    for (int s = sb; s < se; s++) {
        const bool more = s + 1 < se;
        int4 hn = make_int4(0, 0, 0, 0);
        int twn = 0, lenn = 0;
        if (more) {
            hn = P.seg_hdr[s + 1];
            twn = load_tw(P, s + 1, i);
            lenn = kLen ? load_len(P, s + 1, i, hn) : 0;
        }
        float stn = 0.0f;
        auto pre = [&]() {
            if (more) stn = load_stat<MODE, F64>(X, twn, i, hdr_nt(hn));
        };
        TileReg T;
        T.xb = (tw >> 8) * MF_BS;
        T.pr = tile_prec<MODE, F64>(P, tw, st, X);
        if (MODE == MODE_PARITY && !F64) {
            pre();
            if (cnt && i < hdr_nt(h) && chk_in(CHK_TILE, h.x + i, P.ntiles)) {
                const int t = h.x + i;
                atomicAdd(&cnt[T.pr], 1u);
                atomicAdd(&cnt[5 + T.pr], (unsigned)(P.tile_off[t + 1] - P.tile_off[t]));
            }
            acc += slice_dot_parity(P, h, i, hmask, len, T, X);
        } else {
            acc += slice_dot<MODE, F64>(P, h, i, hmask, off, T, X, cnt, pre);
        }
        if (hdr_last(h)) {
            if (chk_in(CHK_ROW, h.y, P.tilem)) epi(h.y, acc);
            acc = 0.0;
        }
        off += (long long)hdr_kp(h) * MF_BS;
        h = hn;
        tw = twn;
        len = lenn;
        st = stn;
    }
}

// ------------------------------------------------------------ phases
struct Ctx {
    int lane, wib, half, i, rbeg, rend, sbeg, send;
    unsigned hmask;
};

__device__ __forceinline__ Ctx make_ctx(const SolverParams &P)
{
    Ctx c;
    c.lane = threadIdx.x & 31;
    c.wib = threadIdx.x >> 5;
    c.half = c.lane >> 4;
    c.i = c.lane & 15;
    c.hmask = 0xFFFFu << (16 * c.half);
    const int hw = (blockIdx.x * kWarps + c.wib) * 2 + c.half;
    c.rbeg = P.hw_begin[hw];
    c.rend = P.hw_begin[hw + 1];
    c.sbeg = P.seg_ptr[c.rbeg];
    c.send = P.seg_ptr[c.rend];
    return c;
}

// max over the 16 lanes of a half-warp; hmask names exactly those lanes (the
// two halves of a warp walk different tile-row ranges, so they never reduce
// together).  One redux.sync instead of a shuffle tree.  half_max takes
// magnitudes (v >= 0), whose IEEE order is the order of their bit patterns.
__device__ __forceinline__ float half_max(float v, unsigned hmask)
{
    return __int_as_float(__reduce_max_sync(hmask, __float_as_int(v)));
}
__device__ __forceinline__ int half_max_i(int v, unsigned hmask)
{
    return __reduce_max_sync(hmask, v);
}

// reference label rank of |dp| (main-cg-mixed.cu:1334-1351): 4 FP64, 3 FP32, 2 FP16, 1 INT8, 0 none
__device__ __forceinline__ int ref_rank(double dp)
{
    if (dp <= 1e-7 && dp > 1e-8) return 1;
    if (dp <= 1e-6 && dp > 1e-7) return 2;
    if (dp <= 1e-5 && dp > 1e-6) return 3;
    if (dp > 1e-5) return 4;
    return 0;
}
__device__ __forceinline__ signed char rank_to_vis(int rank)
{
    // 0 -> bypass(1), 1 -> int8(2), 2 -> fp16(3), 3 -> fp32(4), 4 -> fp64(0)
    return (signed char)(rank == 0 ? 1 : rank == 1 ? 2 : rank == 2 ? 3 : rank == 3 ? 4 : 0);
}

// (int8_t) of a double as the x86-64 host compiler emits it (truncate to int32,
// 0x80000000 when NaN / out of range, keep the low byte) -- the reference
// converts p this way (main-cg-mixed.cu:435).
__device__ __forceinline__ int8_t trunc_i8(double v)
{
    int w;
    if (!(v == v) || v >= 2147483648.0 || v < -2147483648.0) w = (int)0x80000000u;
    else w = (int)v;
    return (int8_t)(unsigned char)(w & 0xFF);
}

// Write a direction vector's shadows and segment statistics for the rows of
// tile-row R (all 16 lanes of the half-warp call this together).
template <int MODE>
__device__ __forceinline__ void publish_dir(int R, int row, bool valid, double vnew, double vold, float *v32,
                                            __half *v16, int8_t *v8, float *mag, signed char *lab, float &bmax,
                                            unsigned hmask, bool labels, float *bmin = nullptr,
                                            float small_thr = -1.0f, float *nsmall = nullptr)
{
    if (MODE == MODE_PARITY && valid) v32[row] = (float)vnew;
    if (MODE == MODE_MIXED) {
        float m = half_max(valid ? (float)fabs(vnew) : 0.0f, hmask);
        bmax = fmaxf(bmax, m);
        if (bmin) *bmin = fminf(*bmin, m);
        // segments at or below small_thr (demote_fp16 x the operand's previous maximum)
        if (nsmall && (threadIdx.x & 15) == 0 && m <= small_thr) *nsmall += 1.0f;
        if ((threadIdx.x & 15) == 0) mag[R] = m;
    } else if (MODE == MODE_PARITY) {
        if (valid) {
            v16[row] = __double2half(vnew);
            v8[row] = trunc_i8(vnew);
        }
        if (labels) {
            // reference rule: label of the next SpMV's tile column from |v_new - v_old|
            int rk = half_max_i(valid ? ref_rank(fabs(vnew - vold)) : 0, hmask);
            if ((threadIdx.x & 15) == 0) lab[R] = rank_to_vis(rk);
        }
    }
}

__device__ __forceinline__ XVec make_x(const double *x64, const float *x32, const __half *x16, const int8_t *x8,
                                       const float *mag, const signed char *lab, float invM, int dyn = 1)
{
    XVec X;
    X.x64 = x64;
    X.x32 = x32;
    X.x16 = x16;
    X.x8 = x8;
    X.mag = mag;
    X.lab = lab;
    X.invM = invM;
    X.force_pr = -1;
    X.dyn = dyn;
    X.lean_pr = MF_P32;
    return X;
}

__device__ __forceinline__ XVec fp64_x(const double *x64)
{
    XVec X = make_x(x64, nullptr, nullptr, nullptr, nullptr, nullptr, 0.f);
    X.force_pr = MF_P64;
    return X;
}

// LB = minimum resident blocks per SM the register budget is sized for:
// 1 -> up to 128 registers (no spills, 16 warps / SM), 2 -> 64 registers (32 warps / SM).
// Block 0 / thread 0 splits its wall time into phases (%globaltimer deltas);
// the state lives in shared memory so the other threads spend no registers on it.
struct PhaseClock {
    Shared *sh;
    __device__ bool on() const { return blockIdx.x == 0 && threadIdx.x == 0; }
    __device__ void start(Shared *s)
    {
        sh = s;
        if (on()) {
            sh->clk_t = mf_globaltimer();
            for (int j = 0; j < 5; j++) sh->clk_acc[j] = 0ull;
        }
    }
    __device__ void lap(int ph)
    {
        if (on()) {
            const unsigned long long n = mf_globaltimer();
            sh->clk_acc[ph] += n - sh->clk_t;
            sh->clk_t = n;
        }
    }
};
enum { PH_SPMV = 0, PH_VECB = 1, PH_VECC = 2, PH_BAR = 3, PH_REPL = 4 };

// After an FP64 residual replacement r = b - A x: keep the CG direction only
// while the recursive residual still told the truth.  When the replacement
// follows a failed convergence check (the recursive residual claimed
// convergence, the true one did not) or the two squared norms differ by more
// than 4x, the recursive residual has drifted to the accuracy floor of the
// low-precision products; beta = r_true.r_true / r_old.r_old would then be
// meaningless (huge when r_old has collapsed), so CG restarts from the true
// residual (beta = 0, which also makes q = A p consistent again).
__device__ __forceinline__ bool restart_after_replacement(bool failed_check, double rr_true, double rr_rec)
{
    return failed_check || rr_true > 4.0 * rr_rec || 4.0 * rr_true < rr_rec;
}

// Relaxed matvec precision (mixed CG): inexact Krylov theory (van den Eshof &
// Sleijpen, SIAM J. Matrix Anal. Appl. 26(1), 2004; Bouras & Fraysse, SIAM J.
// Matrix Anal. Appl. 26(3), 2005) lets the relative error of the product at
// iteration k grow like eps_k = eta * tol / (||r_k|| / ||b||): the further the
// solve has converged, the coarser the operator may be.  The whole SpMV then
// runs in the narrowest stored precision whose rounding stays below eps_k:
// FP16 (unit roundoff 2^-11) when every tile fits FP16's normal range and,
// when allowed, scaled INT8 (half a step of the tile's largest magnitude /
// 127, below 2^-8 of it).  The FP64 residual replacement and the convergence
// test on the FP64 true residual keep the final accuracy either way.
constexpr double kRoundF16 = 1.0 / 2048.0;
constexpr double kRoundI8 = 1.0 / 256.0;
__device__ __forceinline__ int relaxed_precision(const SolverParams &P, double rr, double bb)
{
    if (P.relax_eta <= 0.0f || !(bb > 0.0) || !(rr > 0.0)) return MF_P32;
    const double eps = (double)P.relax_eta * P.tol / sqrt(rr / bb);
    if (P.relax_int8 && eps >= kRoundI8) return MF_P8;
    if (eps >= kRoundF16 && P.fp16_ok) return MF_P16;
    return MF_P32;
}

// METH: MF_METHOD_CG or MF_METHOD_BICGSTAB.  One instantiation per method, so
// each gets its own register allocation: the kernel sits at the 64-register
// limit of two 512-thread blocks per SM, and code in one method's branch
// moves spills into the other's hot loop.
template <int MODE, int LB, int METH>
__global__ void __launch_bounds__(kThreads, LB) k_solve(SolverParams P)
{
    __shared__ Shared sh;
    const Ctx c = make_ctx(P);
    unsigned epoch = 0;
    // tile-use counters: FP64 mode needs none (every tile of every SpMV is FP64;
    // the host derives the totals from the SpMV count)
    unsigned *cnt = (MODE == MODE_FP64) ? nullptr : sh.cnt[c.wib * 2 + c.half];
    if (cnt && c.i < 10) cnt[c.i] = 0u;
    int nspmv = 0;
    __syncwarp();
    PhaseClock clk;
    clk.start(&sh);
    const int n = P.n;
    constexpr bool bicg = (METH == MF_METHOD_BICGSTAB);

    // ---- init: x = 0 (owned rows), r = b, p = r (rh = r) ----
    // With an initial guess: r = b - A x in FP64, and |b|^2 reduced on its own
    // first (it scales the convergence test).
    double pb = 0.0, bb0 = 0.0;
    float bmax = 0.0f, bmin = 3.0e38f, nsm = 0.0f;   // no previous maximum: nothing counts as small
    if (P.x0_given) {
        double pbb = 0.0;
        for (int R = c.rbeg; R < c.rend; R++) {
            const int row = R * MF_BS + c.i;
            if (row < n) pbb += P.b[row] * P.b[row];
        }
        block_partial(P, sh, 8, pbb, 0, 0, 0, 1, 0u);
        if (!grid_barrier(P, epoch, sh)) return;
        double vb[4] = {0.0, 0.0, 0.0, 0.0};
        grid_collect(P, sh, 8, 1, 0u, vb);
        bb0 = vb[0];
        auto init_row = [&](int R, double y) {
            const int row = R * MF_BS + c.i;
            const bool valid = row < n;
            const double rv = valid ? P.b[row] - y : 0.0;
            if (valid) {
                P.r[row] = rv;
                P.p[row] = rv;
                if (bicg) P.rh[row] = rv;
            }
            publish_dir<MODE>(R, row, valid, rv, 0.0, P.p32, P.p16, P.p8, P.mag_p, P.lab_p, bmax, c.hmask, false,
                              &bmin);
            pb += rv * rv;
        };
        spmv_range<MODE, true>(P, c.sbeg, c.send, c.i, c.hmask, fp64_x(P.x), nullptr, init_row);
        for (int R = c.rbeg; R < c.rend; R++)
            if (P.seg_ptr[R] == P.seg_ptr[R + 1]) init_row(R, 0.0);
        nspmv++;
    } else {
        for (int R = c.rbeg; R < c.rend; R++) {
            const int row = R * MF_BS + c.i;
            const bool valid = row < n;
            const double bv = valid ? P.b[row] : 0.0;
            if (valid) {
                P.x[row] = 0.0;
                P.r[row] = bv;
                P.p[row] = bv;
                if (bicg) P.rh[row] = bv;
            }
            // parity mode: labels start all FP64 (cudaMemset(d_vis, 0), main-cg-mixed.cu:2828)
            publish_dir<MODE>(R, row, valid, bv, 0.0, P.p32, P.p16, P.p8, P.mag_p, P.lab_p, bmax, c.hmask, false,
                              &bmin);
            pb += bv * bv;
        }
    }
    // the smallest segment magnitude (carried as -min) matters only to the mixed
    // mode's SpMV; FP64 and parity reduce (sum, max) as before
    // (sum, max, -min, small segments) in mixed mode; FP64 and parity reduce (sum, max)
    constexpr int kNvSeg = (MODE == MODE_MIXED) ? 4 : 2;
    constexpr int kNvSegB = (MODE == MODE_MIXED) ? 3 : 1;      // (max, -min, small) without a sum
    block_partial(P, sh, 0, pb, (double)bmax, -(double)bmin, (double)nsm, kNvSeg, 0x6u);
    if (!grid_barrier(P, epoch, sh)) return;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    grid_collect(P, sh, 0, kNvSeg, 0x6u, v);
    // mixed: can any tile of the next SpMV leave FP32 at all?  Not when the
    // smallest column segment is within demote_fp16 of the largest and no tile
    // is exact in a narrower type: then the SpMV skips its precision lookups.
    // And narrower tiles are considered only when enough segments were small
    // (demote_min_fraction): a few demoted tiles save fewer bytes than the
    // lookups cost in a latency-bound SpMV.
    auto dyn_of = [&](double mx, double neg_mn, double nsmall) -> int {
        return (P.lossless_any ||
                ((mx <= 0.0 || -neg_mn <= (double)P.demote16 * mx) && nsmall >= (double)P.min_small)) ? 1 : 0;
    };
    int dynA = (MODE == MODE_MIXED) ? dyn_of(v[1], v[2], v[3]) : 0;
    // Feedback on the per-slice lookups (mixed BiCGSTAB): each SpMV's reduction
    // also carries how many tiles it ran below FP32.  A dynamic SpMV that
    // demoted fewer than min_demoted (demote_min_fraction of the tiles) did
    // not pay for its lookups, and the same operand's next kDemoteCool SpMVs
    // run the lean walk.  (A slice demotes only when all of its tiles'
    // segments are small: on the 96^3 BiCGSTAB system 1.3 % of the tile
    // products ran below FP32 while the lookups cost 7 % of the solve.)  CG
    // goes without it: the extra reduction value and counters cost its mixed
    // 128^3 solve 3.5 % although its lookups never engage there.
    constexpr bool kFb = (MODE == MODE_MIXED) && bicg;
    constexpr int kNvFb = kFb ? 2 : 1;
    auto demoted = [&]() -> unsigned { return (kFb && c.i == 0) ? cnt[MF_P16] + cnt[MF_P8] : 0u; };
    auto next_cool = [&](int cool, bool was_dyn, double dem) -> int {
        return cool > 0 ? cool - 1 : (was_dyn && dem < (double)P.min_demoted) ? kDemoteCool : 0;
    };
    int coolA = 0, coolS = 0;
    // the base precision of the lookup-free walk (FP16 when every tile is exact in it)
    auto lean_base = [&](XVec X) -> XVec {
        if (P.lean_f16) X.lean_pr = MF_P16;
        return X;
    };
    // mixed CG: the x / r update records r's per-segment magnitudes (one
    // half-warp max reduction and one store per tile-row, 4.5 % of the 128^3
    // solve) only while enough segments were small in the last update that the
    // next SpMV may demote tiles; otherwise it keeps just r's maximum and the
    // count of small segments (a vote per tile-row, on every 4th update only:
    // 1.5 % of the solve when taken on every one), and the next SpMV runs
    // all-FP32.  Demotion then starts up to four updates after the small
    // segments do.
    const float half_small = 0.5f * fmaxf(1.0f, P.min_small);
    int magB = (MODE == MODE_MIXED) ? ((P.lossless_any || v[3] >= (double)half_small) ? 1 : 0) : 1;
            clk.lap(PH_BAR);
    const double bb = P.x0_given ? bb0 : v[0];
    double rr = v[0], r1 = v[0];
    float invM = v[1] > 0.0 ? (float)(1.0 / v[1]) : 0.0f;
    float invMs = 0.0f;
    const double thr2 = P.tol * P.tol * bb;
    int k = 0, conv = 0, repl = 0, status = 0, last_true = 0;
    double rr_true = rr;
    if (!P.fixed_iters && rr <= thr2) { conv = 1; last_true = 1; }

    // tile-rows without slices (all-zero rows) get no SpMV epilogue
    bool has_empty = false;
    for (int R = c.rbeg; R < c.rend && !has_empty; R++) has_empty = P.seg_ptr[R] == P.seg_ptr[R + 1];
    double beta2 = 0.0;
    // mixed CG: uniform reduced precision of the next SpMV (relaxed_precision)
    int prA = (MODE == MODE_MIXED) ? relaxed_precision(P, rr, bb) : MF_P32;

    while (!conv && k < P.max_iter) {
        if (MODE != MODE_PARITY && !bicg) {
            // CG with two grid syncs per iteration.  The SpMV is applied to r:
            // w = A r, then p = r + beta p and q = A p = w + beta q, so p never
            // needs a halo of its own; alpha = r.r / p.q and beta = r'.r' / r.r
            // are the textbook CG scalars (main-cg-mixed.cu:1224-1382 keeps the
            // same formulas with the SpMV on p and a third sync).
            // ---- A: w = A r; p = r + beta p; q = w + beta q; p.q ----
            // (mixed: with a relaxed precision prA the whole SpMV runs in it)
            double ppq = 0.0;
            XVec XA = make_x(P.r, nullptr, nullptr, nullptr, P.mag_r, nullptr, invM, dynA);
            if (MODE == MODE_MIXED && prA != MF_P32) XA.force_pr = prA;
            if (P.lean_f16) XA.lean_pr = MF_P16;
            spmv_range<MODE, false>(P, c.sbeg, c.send, c.i, c.hmask, XA, cnt, [&](int R, double y) {
                const int row = R * MF_BS + c.i;
                if (row < n) {
                    const double pn = P.r[row] + beta2 * P.p[row];
                    const double qn = y + beta2 * P.q[row];
                    P.p[row] = pn;
                    P.q[row] = qn;
                    ppq += pn * qn;
                }
            });
            if (has_empty) {
                for (int R = c.rbeg; R < c.rend; R++) {
                    if (P.seg_ptr[R] != P.seg_ptr[R + 1]) continue;
                    const int row = R * MF_BS + c.i;
                    if (row < n) {
                        const double pn = P.r[row] + beta2 * P.p[row];
                        const double qn = beta2 * P.q[row];
                        P.p[row] = pn;
                        P.q[row] = qn;
                        ppq += pn * qn;
                    }
                }
            }
            nspmv++;
            clk.lap(PH_SPMV);
            block_partial(P, sh, 1, ppq, 0, 0, 0, 1, 0u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 1, 1, 0u, v);
            clk.lap(PH_BAR);
            const double alpha2 = rr / v[0];
            if (!isfinite(alpha2)) { status = MF_ERR_BREAKDOWN; break; }
            // ---- B: x += alpha p; r -= alpha q; r.r; r's shadow ----
            double prr = 0.0;
            float rmax = 0.0f, rmin = 3.0e38f, rsm = 0.0f;
            const float rthr = invM > 0.0f ? P.demote16 / invM : -1.0f;
            const bool voteB = magB || (k & 3) == 0;     // this update counts small segments
            // kVB tile-rows per step: all loads first, so kVB round trips overlap
            for (int R0 = c.rbeg; R0 < c.rend; R0 += kVB) {
                double xv[kVB], pv[kVB], rv[kVB], qv[kVB];
#pragma unroll
                for (int u = 0; u < kVB; u++) {
                    const int row = (R0 + u) * MF_BS + c.i;
                    const bool valid = R0 + u < c.rend && row < n;
                    xv[u] = valid ? P.x[row] : 0.0;
                    pv[u] = valid ? P.p[row] : 0.0;
                    rv[u] = valid ? P.r[row] : 0.0;
                    qv[u] = valid ? P.q[row] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < kVB; u++) {
                    const int R = R0 + u;
                    if (R >= c.rend) break;      // uniform over the half-warp
                    const int row = R * MF_BS + c.i;
                    const bool valid = row < n;
                    const double rn = valid ? rv[u] - alpha2 * qv[u] : 0.0;
                    if (valid) {
                        P.x[row] = xv[u] + alpha2 * pv[u];
                        P.r[row] = rn;
                        prr += rn * rn;
                    }
                    if (MODE != MODE_MIXED || magB) {
                        publish_dir<MODE>(R, row, valid, rn, 0.0, nullptr, nullptr, nullptr, P.mag_r, nullptr, rmax,
                                          c.hmask, false, &rmin, rthr, &rsm);
                    } else {
                        const float m = valid ? (float)fabs(rn) : 0.0f;
                        rmax = fmaxf(rmax, m);
                        if (voteB && __all_sync(c.hmask, m <= rthr) && c.i == 0) rsm += 1.0f;
                    }
                }
            }
            clk.lap(PH_VECB);
            block_partial(P, sh, 2, prr, (double)rmax, -(double)rmin, (double)rsm, kNvSeg, 0x6u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 2, kNvSeg, 0x6u, v);
            clk.lap(PH_BAR);
            double rr_new = v[0];
            const double rr_rec = rr_new;       // recursive r.r of this iteration
            invM = v[1] > 0.0 ? (float)(1.0 / v[1]) : 0.0f;
            if (MODE == MODE_MIXED) {
                dynA = magB ? dyn_of(v[1], v[2], v[3]) : 0;
                if (voteB) magB = (P.lossless_any || v[3] >= (double)half_small) ? 1 : 0;
            }
            k++;
            last_true = 0;
            const bool want_check = !P.fixed_iters && rr_new <= thr2;
            const bool want_repl = P.replace_every > 0 && (k % P.replace_every) == 0;
            bool restart = false;
            if (want_check || want_repl) {
                // ---- FP64 true residual r = b - A x (x is current), r's shadow ----
                double prt = 0.0;
                rmax = 0.0f;
                rmin = 3.0e38f;
                rsm = 0.0f;
                spmv_range<MODE, true>(P, c.sbeg, c.send, c.i, c.hmask, fp64_x(P.x), nullptr,
                                       [&](int R, double y) {
                                           const int row = R * MF_BS + c.i;
                                           const bool valid = row < n;
                                           double rv = 0.0;
                                           if (valid) {
                                               rv = P.b[row] - y;
                                               P.r[row] = rv;
                                               prt += rv * rv;
                                           }
                                           publish_dir<MODE>(R, row, valid, rv, 0.0, nullptr, nullptr, nullptr,
                                                             P.mag_r, nullptr, rmax, c.hmask, false, &rmin,
                                                             rthr, &rsm);
                                       });
                if (has_empty) {
                    for (int R = c.rbeg; R < c.rend; R++) {
                        if (P.seg_ptr[R] != P.seg_ptr[R + 1]) continue;
                        const int row = R * MF_BS + c.i;
                        const bool valid = row < n;
                        const double rv = valid ? P.b[row] : 0.0;
                        if (valid) {
                            P.r[row] = rv;
                            prt += rv * rv;
                        }
                        publish_dir<MODE>(R, row, valid, rv, 0.0, nullptr, nullptr, nullptr, P.mag_r, nullptr, rmax,
                                          c.hmask, false, &rmin, rthr, &rsm);
                    }
                }
                clk.lap(PH_REPL);
                block_partial(P, sh, 5, prt, (double)rmax, -(double)rmin, (double)rsm, kNvSeg, 0x6u);
                if (!grid_barrier(P, epoch, sh)) return;
                grid_collect(P, sh, 5, kNvSeg, 0x6u, v);
                clk.lap(PH_BAR);
                rr_new = v[0];
                invM = v[1] > 0.0 ? (float)(1.0 / v[1]) : 0.0f;
                if (MODE == MODE_MIXED) {
                    dynA = dyn_of(v[1], v[2], v[3]);     // the replacement records every segment
                    magB = (P.lossless_any || v[3] >= (double)half_small) ? 1 : 0;
                }
                rr_true = rr_new;
                repl++;
                last_true = 1;
                if (!P.fixed_iters && rr_new <= thr2) { rr = rr_new; conv = 1; break; }
                restart = restart_after_replacement(want_check, rr_new, rr_rec);
            }
            beta2 = restart ? 0.0 : rr_new / rr;
            rr = rr_new;
            if (MODE == MODE_MIXED) prA = relaxed_precision(P, rr, bb);
            continue;
        }
        double alpha = 0.0, omega = 0.0;
        if (!bicg) {
            // ---- A: q = A p, p.q ----
            double ppq = 0.0;
            spmv_range<MODE, false>(P, c.sbeg, c.send, c.i, c.hmask,
                             make_x(P.p, P.p32, P.p16, P.p8, P.mag_p, P.lab_p, invM), cnt,
                             [&](int R, double y) {
                                 const int row = R * MF_BS + c.i;
                                 if (row < n) {
                                     P.q[row] = y;
                                     ppq += P.p[row] * y;
                                 }
                             });
            nspmv++;
            clk.lap(PH_SPMV);
            block_partial(P, sh, 1, ppq, 0, 0, 0, 1, 0u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 1, 1, 0u, v);
            clk.lap(PH_BAR);
            alpha = rr / v[0];
            if (!isfinite(alpha)) { status = MF_ERR_BREAKDOWN; break; }
            // ---- B: r -= alpha q, r.r  (x is updated with p in phase C) ----
            double prr = 0.0;
            for (int R0 = c.rbeg; R0 < c.rend; R0 += kVB) {
                double rv[kVB], qv[kVB];
#pragma unroll
                for (int u = 0; u < kVB; u++) {
                    const int row = (R0 + u) * MF_BS + c.i;
                    const bool valid = R0 + u < c.rend && row < n;
                    rv[u] = valid ? P.r[row] : 0.0;
                    qv[u] = valid ? P.q[row] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < kVB; u++) {
                    const int row = (R0 + u) * MF_BS + c.i;
                    if (R0 + u < c.rend && row < n) {
                        const double rn = rv[u] - alpha * qv[u];
                        P.r[row] = rn;
                        prr += rn * rn;
                    }
                }
            }
            clk.lap(PH_VECB);
            block_partial(P, sh, 2, prr, 0, 0, 0, 1, 0u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 2, 1, 0u, v);
            clk.lap(PH_BAR);
        } else {
            // ---- BiCGSTAB A1: v = A p, alpha = r1 / (rh.v) ----
            double prv = 0.0;
            const int useA = (kFb && coolA > 0) ? 0 : dynA;
            const unsigned d0A = demoted();
            spmv_range<MODE, false>(P, c.sbeg, c.send, c.i, c.hmask,
                             lean_base(make_x(P.p, P.p32, P.p16, P.p8, P.mag_p, P.lab_p, invM, useA)), cnt,
                             [&](int R, double y) {
                                 const int row = R * MF_BS + c.i;
                                 if (row < n) {
                                     P.q[row] = y;
                                     prv += P.rh[row] * y;
                                 }
                             });
            nspmv++;
            clk.lap(PH_SPMV);
            block_partial(P, sh, 1, prv, (double)(demoted() - d0A), 0, 0, kNvFb, 0u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 1, kNvFb, 0u, v);
            clk.lap(PH_BAR);
            if (kFb) coolA = next_cool(coolA, useA != 0, v[1]);
            alpha = r1 / v[0];
            if (!isfinite(alpha)) { status = MF_ERR_BREAKDOWN; break; }
            // ---- B1: s = r - alpha v ----
            float smax = 0.0f, smin = 3.0e38f, ssm = 0.0f;
            const float sthr = invMs > 0.0f ? P.demote16 / invMs : -1.0f;
            for (int R = c.rbeg; R < c.rend; R++) {
                const int row = R * MF_BS + c.i;
                const bool valid = row < n;
                double sold = 0.0, sn = 0.0;
                if (valid) {
                    sold = P.s[row];
                    sn = P.r[row] - alpha * P.q[row];
                    P.s[row] = sn;
                }
                publish_dir<MODE>(R, row, valid, sn, sold, P.s32, P.s16, P.s8, P.mag_s, P.lab_s, smax, c.hmask,
                                  true, &smin, sthr, &ssm);
            }
            clk.lap(PH_VECB);
            // (max, -min) of s's segment magnitudes; only the mixed mode uses the minimum
            block_partial(P, sh, 2, (double)smax, -(double)smin, (double)ssm, 0, kNvSegB, 0x3u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 2, kNvSegB, 0x3u, v);
            clk.lap(PH_BAR);
            invMs = v[0] > 0.0 ? (float)(1.0 / v[0]) : 0.0f;
            const int dynS = (MODE == MODE_MIXED) ? dyn_of(v[0], v[1], v[2]) : 1;
            // ---- A2: t = A s, omega = (t.s)/(t.t) ----
            double pts = 0.0, ptt = 0.0;
            const int useS = (kFb && coolS > 0) ? 0 : dynS;
            const unsigned d0S = demoted();
            spmv_range<MODE, false>(P, c.sbeg, c.send, c.i, c.hmask,
                             lean_base(make_x(P.s, P.s32, P.s16, P.s8, P.mag_s, P.lab_s, invMs, useS)), cnt,
                             [&](int R, double y) {
                                 const int row = R * MF_BS + c.i;
                                 if (row < n) {
                                     P.t[row] = y;
                                     pts += y * P.s[row];
                                     ptt += y * y;
                                 }
                             });
            nspmv++;
            clk.lap(PH_SPMV);
            block_partial(P, sh, 3, pts, ptt, (double)(demoted() - d0S), 0, kNvFb + 1, 0u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 3, kNvFb + 1, 0u, v);
            clk.lap(PH_BAR);
            if (kFb) coolS = next_cool(coolS, useS != 0, v[2]);
            omega = (v[1] != 0.0) ? v[0] / v[1] : 0.0;
            // ---- B2: x += alpha p + omega s; r = s - omega t ----
            double prr = 0.0, prh = 0.0;
#pragma unroll 2
            for (int R = c.rbeg; R < c.rend; R++) {
                const int row = R * MF_BS + c.i;
                if (row < n) {
                    const double sv = P.s[row];
                    P.x[row] = P.x[row] + alpha * P.p[row] + omega * sv;
                    const double rv = sv - omega * P.t[row];
                    P.r[row] = rv;
                    prr += rv * rv;
                    prh += rv * P.rh[row];
                }
            }
            clk.lap(PH_VECB);
            block_partial(P, sh, 4, prr, prh, 0, 0, 2, 0u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 4, 2, 0u, v);
            clk.lap(PH_BAR);
        }
        double rr_new = v[0], r1_new = bicg ? v[1] : 0.0;
        const double rr_rec = rr_new;    // recursive r.r of this iteration
        k++;
        last_true = 0;
        bool x_done = bicg;      // CG defers x += alpha p to phase C
        const bool want_check = !P.fixed_iters && rr_new <= thr2;
        const bool want_repl = P.replace_every > 0 && (k % P.replace_every) == 0;
        bool restart = false;
        if (want_check || want_repl) {
            if (!x_done) {
                // the FP64 residual needs the current x: apply this iteration's step first
                for (int R = c.rbeg; R < c.rend; R++) {
                    const int row = R * MF_BS + c.i;
                    if (row < n) P.x[row] += alpha * P.p[row];
                }
                x_done = true;
                if (!grid_barrier(P, epoch, sh)) return;
            }
            // ---- FP64 true residual: r = b - A x ----
            double prt = 0.0, prth = 0.0;
            spmv_range<MODE, true>(P, c.sbeg, c.send, c.i, c.hmask, fp64_x(P.x), nullptr, [&](int R, double y) {
                const int row = R * MF_BS + c.i;
                if (row < n) {
                    const double rv = P.b[row] - y;
                    P.r[row] = rv;
                    prt += rv * rv;
                    if (bicg) prth += rv * P.rh[row];
                }
            });
            // rows of tile-rows without tiles (A row = 0): r = b there
            for (int R = c.rbeg; R < c.rend; R++) {
                if (P.seg_ptr[R] != P.seg_ptr[R + 1]) continue;
                const int row = R * MF_BS + c.i;
                if (row < n) {
                    const double rv = P.b[row];
                    P.r[row] = rv;
                    prt += rv * rv;
                    if (bicg) prth += rv * P.rh[row];
                }
            }
            clk.lap(PH_REPL);
            block_partial(P, sh, 5, prt, prth, 0, 0, 2, 0u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 5, 2, 0u, v);
            clk.lap(PH_BAR);
            rr_new = v[0];
            r1_new = v[1];
            rr_true = rr_new;
            repl++;
            last_true = 1;
            if (!P.fixed_iters && rr_new <= thr2) { rr = rr_new; conv = 1; break; }
            restart = restart_after_replacement(want_check, rr_new, rr_rec);
        }
        // ---- C: (CG: x += alpha p,) p = r + beta p  /  p = r + beta (p - omega v) ----
        // A restart (see restart_after_replacement) takes p = r; BiCGSTAB also
        // takes the true residual as its new shadow residual (rh = r, r1 = r.r).
        double beta;
        if (restart) {
            beta = 0.0;
            if (bicg) r1 = rr_new;
        } else if (!bicg) {
            beta = rr_new / rr;
        } else {
            beta = (r1_new * alpha) / (r1 * omega);
            r1 = r1_new;
            if (!isfinite(beta)) { rr = rr_new; status = MF_ERR_BREAKDOWN; break; }
        }
        rr = rr_new;
        bmax = 0.0f;
        float pmin = 3.0e38f, psm = 0.0f;
        const float pthr = invM > 0.0f ? P.demote16 / invM : -1.0f;
        for (int R0 = c.rbeg; R0 < c.rend; R0 += kVB) {
            double pv[kVB], rv[kVB], xq[kVB];    // xq: x (CG, x not yet updated) or v (BiCGSTAB)
#pragma unroll
            for (int u = 0; u < kVB; u++) {
                const int row = (R0 + u) * MF_BS + c.i;
                const bool valid = R0 + u < c.rend && row < n;
                pv[u] = valid ? P.p[row] : 0.0;
                rv[u] = valid ? P.r[row] : 0.0;
                xq[u] = (valid && (bicg || !x_done)) ? (bicg ? P.q[row] : P.x[row]) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < kVB; u++) {
                const int R = R0 + u;
                if (R >= c.rend) break;          // uniform over the half-warp
                const int row = R * MF_BS + c.i;
                const bool valid = row < n;
                const double pold = pv[u];
                const double pn = bicg ? rv[u] + beta * (pold - omega * xq[u]) : rv[u] + beta * pold;
                if (valid) {
                    if (!bicg && !x_done) P.x[row] = xq[u] + alpha * pold;
                    P.p[row] = pn;
                    if (bicg && restart) P.rh[row] = rv[u];
                }
                publish_dir<MODE>(R, row, valid, valid ? pn : 0.0, pold, P.p32, P.p16, P.p8, P.mag_p, P.lab_p,
                                  bmax, c.hmask, true, &pmin, pthr, &psm);
            }
        }
        clk.lap(PH_VECC);
        block_partial(P, sh, 6, (double)bmax, -(double)pmin, (double)psm, 0, kNvSegB, 0x3u);
        if (!grid_barrier(P, epoch, sh)) return;
        grid_collect(P, sh, 6, kNvSegB, 0x3u, v);
            clk.lap(PH_BAR);
        invM = v[0] > 0.0 ? (float)(1.0 / v[0]) : 0.0f;
        if (MODE == MODE_MIXED) dynA = dyn_of(v[0], v[1], v[2]);
    }
    // ---- final FP64 true residual when the last one was not already formed ----
    if (!last_true) {
        double prt = 0.0;
        spmv_range<MODE, true>(P, c.sbeg, c.send, c.i, c.hmask, fp64_x(P.x), nullptr, [&](int R, double y) {
            const int row = R * MF_BS + c.i;
            if (row < n) {
                const double d = P.b[row] - y;
                prt += d * d;
            }
        });
        for (int R = c.rbeg; R < c.rend; R++) {
            if (P.seg_ptr[R] != P.seg_ptr[R + 1]) continue;
            const int row = R * MF_BS + c.i;
            if (row < n) prt += P.b[row] * P.b[row];
        }
        block_partial(P, sh, 7, prt, 0, 0, 0, 1, 0u);
        if (!grid_barrier(P, epoch, sh)) return;
        grid_collect(P, sh, 7, 1, 0u, v);
            clk.lap(PH_BAR);
        rr_true = v[0];
    }
    // tile-use counters
    __syncwarp();
    if (cnt && c.i < 10 && cnt[c.i]) atomicAdd(&P.counts[c.i], (unsigned long long)cnt[c.i]);
    if (clk.on() && P.phase_ns)
        for (int j = 0; j < 5; j++) P.phase_ns[j] = sh.clk_acc[j];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.out[0] = (double)k;
        P.out[1] = (double)conv;
        P.out[2] = bb > 0 ? sqrt(rr_true / bb) : 0.0;
        P.out[3] = bb > 0 ? sqrt(rr / bb) : 0.0;
        P.out[4] = sqrt(rr);
        P.out[5] = (double)repl;
        P.out[6] = (double)status;
        P.out[7] = (double)nspmv;
    }
}

// ------------------------------------------------------------ standalone SpMV
// y = A x, one half-warp per tile-row range (same pipeline as the solver).
template <int MODE, int LB>
__global__ void __launch_bounds__(kThreads, LB) k_spmv(SolverParams P, int force_pr, double *y, int rows_per_hw)
{
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, half = lane >> 4, i = lane & 15;
    const unsigned hmask = 0xFFFFu << (16 * half);
    const int hw = (blockIdx.x * kWarps + wib) * 2 + half;
    const int rb = min(P.tilem, hw * rows_per_hw), re = min(P.tilem, rb + rows_per_hw);
    if (rb >= re) return;
    XVec X = make_x(P.x, P.p32, nullptr, nullptr, nullptr, nullptr, 0.f);
    X.force_pr = force_pr;
    const int n = P.n;
    spmv_range<MODE, MODE == MODE_FP64>(P, P.seg_ptr[rb], P.seg_ptr[re], i, hmask, X, nullptr,
                                        [&](int R, double v) {
        const int row = R * MF_BS + i;
        if (row < n) y[row] = v;
    });
    for (int R = rb; R < re; R++) {          // tile-rows without tiles: y = 0
        if (P.seg_ptr[R] != P.seg_ptr[R + 1]) continue;
        const int row = R * MF_BS + i;
        if (row < n) y[row] = 0.0;
    }
}

// Partition tile-rows over half-warps by the cost prefix (lower bound).
__global__ void k_partition(const long long *__restrict__ cost, int tilem, int nhw, int *__restrict__ hw_begin)
{
    for (int h = blockIdx.x * blockDim.x + threadIdx.x; h <= nhw; h += gridDim.x * blockDim.x) {
        if (h == nhw) { hw_begin[h] = tilem; continue; }
        const long long total = cost[tilem];
        const long long target = (long long)((double)total * (double)h / (double)nhw);
        int lo = 0, hi = tilem;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (cost[mid] < target) lo = mid + 1; else hi = mid;
        }
        hw_begin[h] = lo;
    }
}

__global__ void k_ref_labels(const double *pold, const double *pnew, int nseg, int *vis)
{
    const int lane = threadIdx.x & 31;
    const int half = lane >> 4, i = lane & 15;
    const int seg = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 2 + half;
    const bool valid = seg < nseg;
    const int rk = valid ? ref_rank(fabs(pnew[(long long)seg * MF_BS + i] - pold[(long long)seg * MF_BS + i])) : 0;
    const int m = half_max_i(rk, 0xFFFFu << (16 * half));
    if (valid && i == 0) vis[seg] = rank_to_vis(m);
}

// ------------------------------------------------------------ several right-hand sides
// CG on NR right-hand sides at once (FP64 and mixed modes): the vectors are
// interleaved (row i's NR values contiguous), so every matrix entry is read
// once per SpMV for all NR columns and one grid sync serves every column; the
// scalars alpha_k, beta_k and the convergence state are per column.  Same
// two-sync schedule as the single-column kernel (SpMV on R; P = R + beta P,
// Q = W + beta Q; then X += alpha P, R -= alpha Q).
constexpr int kMaxNR = 8;
constexpr int kRedWidthM = kMaxNR + 2;    // NR dot products + segment max / -min

struct SharedM {
    double wred[kWarps][kRedWidthM];
    double bcast[kRedWidthM];
    double alpha[kMaxNR], beta[kMaxNR], rr[kMaxNR], thr2[kMaxNR], bb[kMaxNR];
    int active[kMaxNR], pending[kMaxNR], iters[kMaxNR], conv[kMaxNR];
    int brk;                  // some column broke down (a scalar became non-finite)
    int flag;                 // grid_barrier's result
};

struct MultiParams {
    const double *B;          // [vec_len * NR] interleaved right-hand sides (zero columns past nr)
    double *X, *R, *Pv, *Q;   // interleaved
    float *mag;               // per tile-row: max over its rows and columns of |R|
    double *red;              // [kinds][G][kRedWidthM]
    double *out;              // per column: iterations, converged, true rel. residual, recursive; then k, status
    int nr;                   // columns in use
};

// Block partial of NV values (maxmask bit k: max instead of sum) into
// red[kind][bidx][*] of an nblk-block group (the grid, or a batched item's team).
template <int NV>
__device__ void block_partial_m(const MultiParams &M, SharedM &sh, int kind, const double (&v)[NV], unsigned maxmask,
                                int nblk, int bidx)
{
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double a = v[k];
        const bool mx = (maxmask >> k) & 1u;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const double b = __shfl_xor_sync(0xffffffffu, a, o);
            a = mx ? fmax(a, b) : a + b;
        }
        if (lane == 0) sh.wred[wib][k] = a;
    }
    __syncthreads();
    // warp w reduces value w (fixed order)
    if (wib < NV) {
        const bool mx = (maxmask >> wib) & 1u;
        double a = (lane < kWarps) ? sh.wred[lane][wib] : (mx ? -1.0e300 : 0.0);
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const double b = __shfl_xor_sync(0xffffffffu, a, o);
            a = mx ? fmax(a, b) : a + b;
        }
        if (lane == 0) M.red[((long long)kind * nblk + bidx) * kRedWidthM + wib] = a;
    }
}

// After the sync: every block of the group sums the nblk partials of `kind` in
// the same order.
template <int NV>
__device__ void grid_collect_m(const MultiParams &M, SharedM &sh, int kind, unsigned maxmask, double (&out)[NV],
                               int nblk)
{
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    if (wib < NV) {
        const bool mx = (maxmask >> wib) & 1u;
        const double id = mx ? -1.0e300 : 0.0;
        double a = id;
        // lane c takes blocks c, c + 32, ...; a pass issues all its loads first
        constexpr int kU = 5;               // 160 blocks per pass (one block per SM on 148 SMs)
        for (int c0 = 0; c0 < nblk; c0 += 32 * kU) {
            double t[kU];
#pragma unroll
            for (int j = 0; j < kU; j++) {
                const int cb = c0 + lane + 32 * j;
                t[j] = cb < nblk ? M.red[((long long)kind * nblk + cb) * kRedWidthM + wib] : id;
            }
#pragma unroll
            for (int j = 0; j < kU; j++) a = mx ? fmax(a, t[j]) : a + t[j];
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const double b = __shfl_xor_sync(0xffffffffu, a, o);
            a = mx ? fmax(a, b) : a + b;
        }
        if (lane == 0) sh.bcast[wib] = a;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; k++) out[k] = sh.bcast[k];
    __syncthreads();
}

// One chunk of the NR-column walk: lane i's stored values of the chunk at
// entry offset cb in precision PR (FP32 / FP16 / scaled INT8 widened to FP64
// against the FP64 operand rows, as the single-column walk: no FP32 copy of
// R), each times its gathered NR-wide operand row.  The values are loaded one
// at a time next to their use: the NR-wide accumulators and operand rows take
// the registers, and these solves wait on the operand rows, not the values.
template <int PR, int NR>
__device__ __forceinline__ void multi_chunk(const SolverParams &P, long long cb, int i, unsigned hmask, int xb, int k0,
                                            int len, float sc, const double *X64, double (&acc)[NR])
{
    const unsigned long long m8 = __ldcs((const unsigned long long *)(P.meta + cb) + i);
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const unsigned mm = (unsigned)(m8 >> (8 * j)) & 0xFFu;
        const int slot = (int)(mm >> 4);
        const int xi = __shfl_sync(hmask, xb, slot, 16) + (int)(mm & 15u);
        const float s8 = (PR == MF_P8) ? __shfl_sync(hmask, sc, slot, 16) : 0.0f;
        if ((NR < 8 || k0 + j < len) && chk_in(CHK_X, xi, P.chk_xlen)) {
            double a;
            if (PR == MF_P64) a = __ldcs(P.v64 + mf_slot<8>(cb, j, i));
            else if (PR == MF_P32) a = (double)__ldcs(P.v32 + mf_slot<4>(cb, j, i));
            else if (PR == MF_P16) a = (double)__half2float(P.v16[mf_slot<2>(cb, j, i)]);
            else a = (double)((float)P.v8[mf_slot<1>(cb, j, i)] * s8);
            if constexpr (NR == 1) {
                acc[0] = fma(a, X64[xi], acc[0]);
            } else {
                const double2 *xr = (const double2 *)(X64 + (long long)xi * NR);
#pragma unroll
                for (int q = 0; q < NR / 2; q++) {
                    const double2 d = xr[q];
                    acc[2 * q] = fma(a, d.x, acc[2 * q]);
                    acc[2 * q + 1] = fma(a, d.y, acc[2 * q + 1]);
                }
            }
        }
    }
}

// Y = A X for NR interleaved columns over the half-warp's slices; epi(R, acc)
// once per tile-row with lane i's NR row sums.  Precision per slice as in
// slice_dot (mixed: from the column segments' max over rows and columns).
// Up to 4 columns the walk reads no row lengths (padding is value 0 with
// index byte 0, as in slice_dot_uniform: measured 10 % faster on the
// 512-system batch); with 8 columns a padding entry would gather 64 bytes of
// X, and the row-length predicate measured 6 % faster on the 512^2 system.
template <int MODE, int NR, bool F64, typename Epi>
__device__ __forceinline__ void spmv_multi(const SolverParams &P, int sb, int se, int i, unsigned hmask,
                                           const double *X64, const float *mag, float invM,
                                           int dyn, Epi epi)
{
    constexpr bool kMixed = (MODE == MODE_MIXED) && !F64;
    constexpr bool kLen = NR >= 8;
    XVec X = make_x(X64, nullptr, nullptr, nullptr, mag, nullptr, invM, dyn);
    double acc[NR];
#pragma unroll
    for (int k = 0; k < NR; k++) acc[k] = 0.0;
    if (sb >= se) return;
    if (!chk_in(CHK_SLICE, sb, P.nseg) || !chk_in(CHK_SLICE, se - 1, P.nseg)) return;
    int4 h = P.seg_hdr[sb];
    int tw = load_tw(P, sb, i);
    int len = kLen ? load_len(P, sb, i, h) : 0;
    for (int s = sb; s < se; s++) {
        const bool more = s + 1 < se;
        int4 hn = make_int4(0, 0, 0, 0);
        int twn = 0, lenn = 0;
        if (more) {
            hn = P.seg_hdr[s + 1];
            twn = load_tw(P, s + 1, i);
            lenn = kLen ? load_len(P, s + 1, i, hn) : 0;
        }
        const int xb = (tw >> 8) * MF_BS;
        int pr = MF_P64;
        if (kMixed && !dyn) {
            pr = MF_P32;                 // no tile can leave FP32 in this SpMV: no lookups
        } else if (kMixed) {
            const float st = (i < hdr_nt(h)) ? mag[tw >> 8] : 0.0f;
            pr = __reduce_min_sync(hmask, (i < hdr_nt(h)) ? tile_prec<MODE, false>(P, tw, st, X) : MF_P8);
        }
        float sc = 0.0f;
        if (kMixed && pr == MF_P8)
            sc = (i < hdr_nt(h) && chk_in(CHK_TILE, h.x + i, P.ntiles)) ? P.i8_scale[h.x + i] : 0.0f;
        const int kp = hdr_kp(h);
        const long long off = hdr_off(h);
        const int kpc = chk_in(CHK_PAYLOAD, off + (long long)kp * MF_BS - 1, P.n_payload) ? kp : 0;
        for (int k0 = 0; k0 < kpc; k0 += 8) {
            const long long cb = off + (long long)(k0 >> 3) * 128;
            // one instantiation per stored precision, so only that precision's
            // values are live across the chunk's gathers
            if (!kMixed || pr == MF_P64) multi_chunk<MF_P64, NR>(P, cb, i, hmask, xb, k0, len, sc, X64, acc);
            else if (pr == MF_P32) multi_chunk<MF_P32, NR>(P, cb, i, hmask, xb, k0, len, sc, X64, acc);
            else if (pr == MF_P16) multi_chunk<MF_P16, NR>(P, cb, i, hmask, xb, k0, len, sc, X64, acc);
            else multi_chunk<MF_P8, NR>(P, cb, i, hmask, xb, k0, len, sc, X64, acc);
        }
        if (hdr_last(h)) {
            if (chk_in(CHK_ROW, h.y, P.tilem)) epi(h.y, acc);
#pragma unroll
            for (int k = 0; k < NR; k++) acc[k] = 0.0;
        }
        h = hn;
        tw = twn;
        len = lenn;
    }
}

// Largest / smallest segment magnitude of the SpMV operand (mixed mode).
struct SegMM {
    float mx, mn;
};

// R's segment magnitude (max over the tile-row's rows and all columns) for
// tile-row R; all 16 lanes of the half-warp call it together.
template <int MODE, int NR>
__device__ __forceinline__ void publish_multi(const MultiParams &M, int R, int row, bool valid, const double (&rv)[NR],
                                              SegMM &st, unsigned hmask)
{
    if (MODE != MODE_MIXED) return;
    float m = 0.0f;
    if (valid) {
#pragma unroll
        for (int q = 0; q < NR; q++) m = fmaxf(m, fabsf((float)rv[q]));
    }
    m = half_max(m, hmask);
    st.mx = fmaxf(st.mx, m);
    st.mn = fminf(st.mn, m);
    if ((threadIdx.x & 15) == 0) M.mag[R] = m;
}

template <int NR>
__device__ __forceinline__ void load_row(const double *v, int row, double (&out)[NR])
{
    if constexpr (NR == 1) {
        out[0] = v[row];
        return;
    }
    const double2 *p = (const double2 *)(v + (long long)row * NR);
#pragma unroll
    for (int q = 0; q < NR / 2; q++) {
        const double2 d = p[q];
        out[2 * q] = d.x;
        out[2 * q + 1] = d.y;
    }
}
template <int NR>
__device__ __forceinline__ void store_row(double *v, int row, const double (&in)[NR])
{
    if constexpr (NR == 1) {
        v[row] = in[0];
        return;
    }
    double2 *p = (double2 *)(v + (long long)row * NR);
#pragma unroll
    for (int q = 0; q < NR / 2; q++) p[q] = make_double2(in[2 * q], in[2 * q + 1]);
}

// The CG iterations on NR columns, generic in how the threads that share a
// system synchronise: the whole grid (k_solve_multi) or one block (k_batch).
template <int MODE, int NR, class Sync>
__device__ void cg_multi_body(const SolverParams &P, const MultiParams &M, const Ctx &c, SharedM &sh, Sync &sy)
{
    const int n = P.n;
    bool has_empty = false;
    for (int R = c.rbeg; R < c.rend && !has_empty; R++) has_empty = P.seg_ptr[R] == P.seg_ptr[R + 1];
    const unsigned mm2 = 3u << NR;          // the two trailing max slots

    // ---- init: X = 0, R = B, P = Q = 0; |b_k|^2; R's segment magnitudes ----
    // With an initial guess (x0_given): |b_k|^2 reduced first (it scales the
    // convergence test), then R = B - A X in FP64.
    double pb[NR + 2], bb0[NR];
#pragma unroll
    for (int k = 0; k < NR + 2; k++) pb[k] = 0.0;
    SegMM st = {0.0f, 3.0e38f};
    if (P.x0_given) {
        double pbb[NR];
#pragma unroll
        for (int k = 0; k < NR; k++) pbb[k] = 0.0;
        for (int R = c.rbeg; R < c.rend; R++) {
            const int row = R * MF_BS + c.i;
            if (row < n) {
                double bv[NR];
                load_row<NR>(M.B, row, bv);
#pragma unroll
                for (int k = 0; k < NR; k++) pbb[k] += bv[k] * bv[k];
            }
        }
        if (!sy.template reduce<NR>(8, pbb, 0u, bb0)) return;
        auto init_r = [&](int R, const double (&y)[NR]) {
            const int row = R * MF_BS + c.i;
            const bool valid = row < n;
            double rv[NR], z[NR];
#pragma unroll
            for (int k = 0; k < NR; k++) { rv[k] = 0.0; z[k] = 0.0; }
            if (valid) {
                load_row<NR>(M.B, row, rv);
#pragma unroll
                for (int k = 0; k < NR; k++) rv[k] -= y[k];
                store_row<NR>(M.R, row, rv);
                store_row<NR>(M.Pv, row, z);
                store_row<NR>(M.Q, row, z);
#pragma unroll
                for (int k = 0; k < NR; k++) pb[k] += rv[k] * rv[k];
            }
            publish_multi<MODE, NR>(M, R, row, valid, rv, st, c.hmask);
        };
        spmv_multi<MODE, NR, true>(P, c.sbeg, c.send, c.i, c.hmask, M.X, nullptr, 0.0f, 1, init_r);
        if (has_empty) {
            double zy[NR];
#pragma unroll
            for (int k = 0; k < NR; k++) zy[k] = 0.0;
            for (int R = c.rbeg; R < c.rend; R++)
                if (P.seg_ptr[R] == P.seg_ptr[R + 1]) init_r(R, zy);
        }
    } else {
        for (int R = c.rbeg; R < c.rend; R++) {
            const int row = R * MF_BS + c.i;
            const bool valid = row < n;
            double rv[NR], z[NR];
#pragma unroll
            for (int k = 0; k < NR; k++) { rv[k] = 0.0; z[k] = 0.0; }
            if (valid) {
                load_row<NR>(M.B, row, rv);
                store_row<NR>(M.X, row, z);
                store_row<NR>(M.R, row, rv);
                store_row<NR>(M.Pv, row, z);
                store_row<NR>(M.Q, row, z);
#pragma unroll
                for (int k = 0; k < NR; k++) pb[k] += rv[k] * rv[k];
            }
            publish_multi<MODE, NR>(M, R, row, valid, rv, st, c.hmask);
        }
    }
    pb[NR] = st.mx;
    pb[NR + 1] = -st.mn;
    double v[NR + 2];
    if (!sy.template reduce<NR + 2>(0, pb, mm2, v)) return;
    if (threadIdx.x == 0) {
        for (int k = 0; k < NR; k++) {
            sh.bb[k] = P.x0_given ? bb0[k] : v[k];
            sh.rr[k] = v[k];
            sh.thr2[k] = P.tol * P.tol * sh.bb[k];
            sh.beta[k] = 0.0;
            sh.pending[k] = 0;
            sh.iters[k] = 0;
            sh.conv[k] = (k < M.nr && !P.fixed_iters && v[k] <= sh.thr2[k]) ? 1 : 0;
            sh.active[k] = (k < M.nr && !sh.conv[k]) ? 1 : 0;
        }
        sh.brk = 0;
    }
    __syncthreads();
    float invM = v[NR] > 0.0 ? (float)(1.0 / v[NR]) : 0.0f;
    // mixed: some tile may leave FP32 only if the smallest segment is below
    // demote_fp16 of the largest or lossless classes apply (see dyn in XVec)
    auto dyn_of = [&](double mx, double neg_mn) -> int {
        return (P.lossless_any || mx <= 0.0 || -neg_mn <= (double)P.demote16 * mx) ? 1 : 0;
    };
    int dyn = dyn_of(v[NR], v[NR + 1]);
    int k = 0, status = 0, repl = 0, last_true = 0;
    double rt[NR];
#pragma unroll
    for (int j = 0; j < NR; j++) rt[j] = v[j];

    for (;;) {
        int any = 0;
#pragma unroll
        for (int j = 0; j < NR; j++) any |= sh.active[j];
        if (!any || k >= P.max_iter) break;
        // ---- A: W = A R; P = R + beta P; Q = W + beta Q; P.Q per column ----
        double ppq[NR];
#pragma unroll
        for (int j = 0; j < NR; j++) ppq[j] = 0.0;
        auto upd_a = [&](int R, const double (&w)[NR]) {
            const int row = R * MF_BS + c.i;
            if (row < n) {
                double r[NR], p[NR], q[NR];
                load_row<NR>(M.R, row, r);
                load_row<NR>(M.Pv, row, p);
                load_row<NR>(M.Q, row, q);
#pragma unroll
                for (int j = 0; j < NR; j++) {
                    p[j] = r[j] + sh.beta[j] * p[j];
                    q[j] = w[j] + sh.beta[j] * q[j];
                    ppq[j] += p[j] * q[j];
                }
                store_row<NR>(M.Pv, row, p);
                store_row<NR>(M.Q, row, q);
            }
        };
        spmv_multi<MODE, NR, false>(P, c.sbeg, c.send, c.i, c.hmask, M.R, M.mag, invM, dyn, upd_a);
        if (has_empty) {
            double zw[NR];
#pragma unroll
            for (int j = 0; j < NR; j++) zw[j] = 0.0;
            for (int R = c.rbeg; R < c.rend; R++)
                if (P.seg_ptr[R] == P.seg_ptr[R + 1]) upd_a(R, zw);
        }
        double pq[NR];
        if (!sy.template reduce<NR>(1, ppq, 0u, pq)) return;
        if (threadIdx.x == 0) {
            for (int j = 0; j < NR; j++) {
                double a = sh.active[j] ? sh.rr[j] / pq[j] : 0.0;
                if (!isfinite(a)) {      // breakdown of this column: it stops where it is
                    a = 0.0;
                    sh.active[j] = 0;
                    sh.brk = 1;
                }
                sh.alpha[j] = a;
            }
        }
        __syncthreads();
        if (sh.brk) status = MF_ERR_BREAKDOWN;
        // ---- B: X += alpha P; R -= alpha Q; R.R; R's shadow ----
        double prr[NR + 2];
#pragma unroll
        for (int j = 0; j < NR + 2; j++) prr[j] = 0.0;
        st = SegMM{0.0f, 3.0e38f};
        for (int R = c.rbeg; R < c.rend; R++) {
            const int row = R * MF_BS + c.i;
            const bool valid = row < n;
            double r[NR];
#pragma unroll
            for (int j = 0; j < NR; j++) r[j] = 0.0;
            if (valid) {
                double x[NR], p[NR], q[NR];
                load_row<NR>(M.X, row, x);
                load_row<NR>(M.Pv, row, p);
                load_row<NR>(M.R, row, r);
                load_row<NR>(M.Q, row, q);
#pragma unroll
                for (int j = 0; j < NR; j++) {
                    x[j] += sh.alpha[j] * p[j];
                    r[j] -= sh.alpha[j] * q[j];
                    prr[j] += r[j] * r[j];
                }
                store_row<NR>(M.X, row, x);
                store_row<NR>(M.R, row, r);
            }
            publish_multi<MODE, NR>(M, R, row, valid, r, st, c.hmask);
        }
        prr[NR] = st.mx;
        prr[NR + 1] = -st.mn;
        if (!sy.template reduce<NR + 2>(2, prr, mm2, v)) return;
        invM = v[NR] > 0.0 ? (float)(1.0 / v[NR]) : 0.0f;
        dyn = dyn_of(v[NR], v[NR + 1]);
        k++;
        last_true = 0;
        bool want_repl = P.replace_every > 0 && (k % P.replace_every) == 0;
#pragma unroll
        for (int j = 0; j < NR; j++)
            if (sh.active[j] && !P.fixed_iters && v[j] <= sh.thr2[j]) want_repl = true;
        double rnew[NR], rrec[NR];
#pragma unroll
        for (int j = 0; j < NR; j++) rnew[j] = rrec[j] = v[j];
        if (want_repl) {
            // ---- FP64 R = B - A X, R's shadow, true residual norms ----
            double prt[NR + 2];
#pragma unroll
            for (int j = 0; j < NR + 2; j++) prt[j] = 0.0;
            st = SegMM{0.0f, 3.0e38f};
            auto upd_r = [&](int R, const double (&y)[NR]) {
                const int row = R * MF_BS + c.i;
                const bool valid = row < n;
                double r[NR];
#pragma unroll
                for (int j = 0; j < NR; j++) r[j] = 0.0;
                if (valid) {
                    load_row<NR>(M.B, row, r);
#pragma unroll
                    for (int j = 0; j < NR; j++) {
                        r[j] -= y[j];
                        prt[j] += r[j] * r[j];
                    }
                    store_row<NR>(M.R, row, r);
                }
                publish_multi<MODE, NR>(M, R, row, valid, r, st, c.hmask);
            };
            spmv_multi<MODE, NR, true>(P, c.sbeg, c.send, c.i, c.hmask, M.X, nullptr, 0.0f, 1, upd_r);
            if (has_empty) {
                double zy[NR];
#pragma unroll
                for (int j = 0; j < NR; j++) zy[j] = 0.0;
                for (int R = c.rbeg; R < c.rend; R++)
                    if (P.seg_ptr[R] == P.seg_ptr[R + 1]) upd_r(R, zy);
            }
            prt[NR] = st.mx;
            prt[NR + 1] = -st.mn;
            if (!sy.template reduce<NR + 2>(5, prt, mm2, v)) return;
            invM = v[NR] > 0.0 ? (float)(1.0 / v[NR]) : 0.0f;
            dyn = dyn_of(v[NR], v[NR + 1]);
            repl++;
            last_true = 1;
#pragma unroll
            for (int j = 0; j < NR; j++) {
                rt[j] = v[j];
                rnew[j] = v[j];
            }
        }
        if (threadIdx.x == 0) {
            for (int j = 0; j < NR; j++) {
                if (sh.active[j] && last_true && !P.fixed_iters && rnew[j] <= sh.thr2[j]) {
                    sh.active[j] = 0;            // converged on the FP64 true residual
                    sh.conv[j] = 1;
                    sh.iters[j] = k;
                }
                const bool restart = last_true &&
                                     restart_after_replacement(!P.fixed_iters && rrec[j] <= sh.thr2[j], rnew[j], rrec[j]);
                sh.beta[j] = (sh.active[j] && !restart) ? rnew[j] / sh.rr[j] : 0.0;
                if (sh.active[j] || !sh.conv[j]) sh.rr[j] = rnew[j];
            }
        }
        __syncthreads();
    }
    // ---- final FP64 true residuals when the last step did not form them ----
    if (!last_true) {
        double prt[NR];
#pragma unroll
        for (int j = 0; j < NR; j++) prt[j] = 0.0;
        auto acc_r = [&](int R, const double (&y)[NR]) {
            const int row = R * MF_BS + c.i;
            if (row < n) {
                double b[NR];
                load_row<NR>(M.B, row, b);
#pragma unroll
                for (int j = 0; j < NR; j++) prt[j] += (b[j] - y[j]) * (b[j] - y[j]);
            }
        };
        spmv_multi<MODE, NR, true>(P, c.sbeg, c.send, c.i, c.hmask, M.X, nullptr, 0.0f, 1, acc_r);
        if (has_empty) {
            double zy[NR];
#pragma unroll
            for (int j = 0; j < NR; j++) zy[j] = 0.0;
            for (int R = c.rbeg; R < c.rend; R++)
                if (P.seg_ptr[R] == P.seg_ptr[R + 1]) acc_r(R, zy);
        }
        double w[NR];
        if (!sy.template reduce<NR>(7, prt, 0u, w)) return;
#pragma unroll
        for (int j = 0; j < NR; j++) rt[j] = w[j];
    }
    if (sy.writer()) {
        for (int j = 0; j < NR; j++) {
            const double bb = sh.bb[j];
            M.out[4 * j + 0] = (double)(sh.conv[j] ? sh.iters[j] : k);
            M.out[4 * j + 1] = (double)sh.conv[j];
            M.out[4 * j + 2] = bb > 0 ? sqrt(rt[j] / bb) : 0.0;
            M.out[4 * j + 3] = bb > 0 ? sqrt(sh.rr[j] / bb) : 0.0;
        }
        M.out[4 * NR + 0] = (double)k;
        M.out[4 * NR + 1] = (double)status;
        M.out[4 * NR + 2] = (double)repl;
    }
}

// Grid-wide synchronisation: block partials, the counter barrier, a fixed-order collect.
struct GridSync {
    const SolverParams &P;
    const MultiParams &M;
    SharedM &sh;
    unsigned epoch;
    template <int NV>
    __device__ bool reduce(int kind, const double (&v)[NV], unsigned maxmask, double (&out)[NV])
    {
        block_partial_m<NV>(M, sh, kind, v, maxmask, (int)gridDim.x, (int)blockIdx.x);
        if (!grid_barrier(P, epoch, sh)) return false;
        grid_collect_m<NV>(M, sh, kind, maxmask, out, (int)gridDim.x);
        return true;
    }
    __device__ bool writer() const { return blockIdx.x == 0 && threadIdx.x == 0; }
};

template <int MODE, int NR>
__global__ void __launch_bounds__(kThreads, 1) k_solve_multi(SolverParams P, MultiParams M)
{
    __shared__ SharedM sh;
    const Ctx c = make_ctx(P);
    GridSync sy{P, M, sh, 0u};
    cg_multi_body<MODE, NR>(P, M, c, sh, sy);
}

// ------------------------------------------------------------ batched systems
// Many independent systems in one persistent launch of one or two 512-thread
// blocks per SM (k_batch<MODE, LB>).  Work items are (system, up to 8 of its
// right-hand sides).
//  * Team items: an item whose estimated cost exceeds a fair share of the
//    launch (total cost / blocks) is solved by a team of k blocks, sized by its
//    cost; the host list-schedules team items onto blocks (the k blocks that
//    are free first) and gives every block its ordered list.  Team members
//    synchronise through a counter of their own (bounded waits) and reduce in
//    a fixed order over the k block partials.
//  * Queue items: everything else sits in a device work queue, largest
//    estimated cost first; a block that has finished its list takes the next
//    queue item and solves it alone with block-level syncs.
// The launch is cooperative, so every block is resident and a team never waits
// on a block that cannot run; the lists are sorted by the same global order
// (scheduled start, then item), so no two teams wait on each other.
constexpr int kHalvesPerBlock = kWarps * 2;
constexpr int kMinTeamRows = 64;  // tile-rows per team block at least (2 per half-warp)
// Team size = round(kTeamGrain x cost / fair share): a team's members finish an
// item in about 1 / kTeamGrain of a fair share, so no single item sets the
// launch's end.  A team costs a few microseconds per sync, small against the
// milliseconds a large item's iteration takes on one block.
// Measured on the 512-system batch: grain 1, 2, 4 -> 20.2, 18.7, 17.8 s.
constexpr double kTeamGrain = 4.0;

struct BatchItem {
    const int *seg_ptr;
    const int4 *seg_hdr;
    const int *seg_tile;
    const uint16_t *seg_rowlen;
    const unsigned char *meta;
    const double *v64;
    const float *v32;
    const __half *v16;
    const int8_t *v8;
    const float *i8_scale;
    const long long *row_cost;    // tile-row cost prefix [tilem + 1]
    MultiParams M;                // the item's interleaved vectors and report words (M.nr columns used);
                                  // team items: M.red holds the team's partials [kinds][team][kRedWidthM]
    unsigned *ctr;                // team items: the team's barrier counter (zeroed before the launch)
    long long n_exact;            // tiles exact in INT8 / FP16
    int n, tilem, nr;             // nr: interleave width (1, 2, 4 or 8)
    int tilenum;
    int team;                     // blocks solving the item (1: queue item)
    int nseg, vec_len;            // extents for the bounds-checked build
    long long n_payload;
};

struct BatchParams {
    const BatchItem *items;
    const int *order;             // queue items, largest estimated cost first
    int n_items;                  // queue items
    int n_all;                    // entries of `items` (queue and team items)
    unsigned *head;               // next position in `order` (zeroed before the launch)
    const int *bptr;              // [grid + 1] each block's list of team entries
    const int2 *blist;            // (item, rank in its team)
    int *err;                     // first error of a team wait (zeroed before the launch)
    unsigned long long timeout_ns, arrive_timeout_ns;
    int stall_first;              // test hook: a team's first barrier expects one extra arrival
    int x0_given;                 // every item's X holds its initial guess
    int max_iter, fixed_iters, replace_every, use_lossless;
    double tol, min_fraction;
    float demote16, demote8;
};

// One block's synchronisation: warp shuffles, shared memory, fixed order.
struct BlockSync {
    SharedM &sh;
    template <int NV>
    __device__ bool reduce(int, const double (&v)[NV], unsigned maxmask, double (&out)[NV])
    {
        const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double a = v[k];
            const bool mx = (maxmask >> k) & 1u;
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                const double b = __shfl_xor_sync(0xffffffffu, a, o);
                a = mx ? fmax(a, b) : a + b;
            }
            if (lane == 0) sh.wred[wib][k] = a;
        }
        __syncthreads();
        if (wib < NV) {
            const bool mx = (maxmask >> wib) & 1u;
            double a = (lane < kWarps) ? sh.wred[lane][wib] : (mx ? -1.0e300 : 0.0);
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                const double b = __shfl_xor_sync(0xffffffffu, a, o);
                a = mx ? fmax(a, b) : a + b;
            }
            if (lane == 0) sh.bcast[wib] = a;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < NV; k++) out[k] = sh.bcast[k];
        __syncthreads();
        return true;
    }
    __device__ bool writer() const { return threadIdx.x == 0; }
};

// Barrier of the k blocks of one team: a monotone counter with the pattern of
// grid_barrier (fence, relaxed add, relaxed polls, one acquire fence), bounded
// by `limit_ns`; a timeout, or an error set elsewhere, returns false and the
// first error is kept in *err.
__device__ bool team_barrier(unsigned *ctr, unsigned k, unsigned &epoch, int *err, unsigned long long limit_ns,
                             SharedM &sh, int stall = 0)
{
    __syncthreads();
    epoch += 1;
    if (threadIdx.x == 0) {
        const unsigned target = epoch * k + ((stall && epoch == 1) ? 1u : 0u);
        __threadfence();
        mf_red_relaxed_add_u32(ctr, 1u);
        bool ok = true;
        const unsigned long long t0 = mf_globaltimer();
        unsigned spins = 0;
        for (;;) {
            const unsigned v = mf_ld_relaxed_u32(ctr);
            if ((int)(v - target) >= 0) break;
            if (*(volatile int *)err) { ok = false; break; }
            if ((++spins & 63u) == 0u && mf_globaltimer() - t0 > limit_ns) {
                atomicCAS(err, 0, MF_ERR_TIMEOUT);
                ok = false;
                break;
            }
        }
        mf_fence_acq_rel_gpu();
        sh.flag = ok ? 1 : 0;
    }
    __syncthreads();
    return sh.flag != 0;
}

// The synchronisation of a team item: block partials into the team's slots,
// the team barrier, then every member sums the k partials in the same order.
// The first barrier (every member arriving at the item) may wait for members
// still finishing earlier list entries, so it gets the longer limit.  The
// team's parameters live in shared memory (no registers held across the body).
struct TeamShared {
    double *red;
    unsigned *ctr;
    int *err;
    unsigned long long limit_ns, arrive_ns;
    int k, r;
    unsigned epoch;
    int stall;
};

struct TeamSync {
    SharedM &sh;
    TeamShared &ts;
    template <int NV>
    __device__ bool reduce(int kind, const double (&v)[NV], unsigned maxmask, double (&out)[NV])
    {
        MultiParams R;
        R.red = ts.red;
        block_partial_m<NV>(R, sh, kind, v, maxmask, ts.k, ts.r);
        unsigned ep = ts.epoch;
        const bool ok =
            team_barrier(ts.ctr, (unsigned)ts.k, ep, ts.err, ep == 0 ? ts.arrive_ns : ts.limit_ns, sh, ts.stall);
        if (!ok) return false;
        grid_collect_m<NV>(R, sh, kind, maxmask, out, ts.k);
        if (threadIdx.x == 0) ts.epoch = ep;
        __syncthreads();
        return true;
    }
    __device__ bool writer() const { return ts.r == 0 && threadIdx.x == 0; }
};

// The half-warps of a team of k blocks (this block: rank r) split a system's
// tile-rows by the cost prefix (k = 1: one block).
__device__ __forceinline__ Ctx team_ctx(const BatchItem &it, int r, int k)
{
    Ctx c;
    c.lane = threadIdx.x & 31;
    c.wib = threadIdx.x >> 5;
    c.half = c.lane >> 4;
    c.i = c.lane & 15;
    c.hmask = 0xFFFFu << (16 * c.half);
    const int halves = kHalvesPerBlock * k;
    const int hw = r * kHalvesPerBlock + c.wib * 2 + c.half;
    const long long total = it.row_cost[it.tilem];
    auto split = [&](int h) -> int {
        if (h >= halves) return it.tilem;
        const long long target = (long long)((double)total * (double)h / (double)halves);
        int lo = 0, hi = it.tilem;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (it.row_cost[mid] < target) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    };
    c.rbeg = split(hw);
    c.rend = split(hw + 1);
    c.sbeg = it.seg_ptr[c.rbeg];
    c.send = it.seg_ptr[c.rend];
    return c;
}

// The fields of SolverParams the CG body and the slice walk read, for one item.
__device__ __forceinline__ SolverParams item_params(const BatchItem &it, const BatchParams &B)
{
    SolverParams P;
    P.n = it.n;
    P.tilem = it.tilem;
    P.seg_ptr = it.seg_ptr;
    P.seg_hdr = it.seg_hdr;
    P.seg_tile = it.seg_tile;
    P.seg_rowlen = it.seg_rowlen;
    P.meta = it.meta;
    P.v64 = it.v64;
    P.v32 = it.v32;
    P.v16 = it.v16;
    P.v8 = it.v8;
    P.i8_scale = it.i8_scale;
    P.max_iter = B.max_iter;
    P.x0_given = B.x0_given;
    P.fixed_iters = B.fixed_iters;
    P.replace_every = B.replace_every;
    P.use_lossless = B.use_lossless;
    P.lossless_any = (B.use_lossless && it.n_exact > 0 && (double)it.n_exact >= B.min_fraction * (double)it.tilenum)
                         ? 1 : 0;
    P.tol = B.tol;
    P.demote16 = B.demote16;
    P.demote8 = B.demote8;
    P.nseg = it.nseg;
    P.ntiles = it.tilenum;
    P.chk_xlen = it.vec_len;
    P.n_payload = it.n_payload;
    return P;
}

// MAXNR: the widest interleave the launch was built for (8 with one block per
// SM; 4 with two, whose items never exceed 4 columns).
template <int MODE, int MAXNR, class Sync>
__device__ __forceinline__ void item_solve(const SolverParams &P, const MultiParams &M, int nr, const Ctx &c,
                                           SharedM &sh, Sync &sy)
{
    switch (nr) {
    case 1: cg_multi_body<MODE, 1>(P, M, c, sh, sy); break;
    case 2: cg_multi_body<MODE, 2>(P, M, c, sh, sy); break;
    case 4: cg_multi_body<MODE, 4>(P, M, c, sh, sy); break;
    default:
        if constexpr (MAXNR >= 8) cg_multi_body<MODE, 8>(P, M, c, sh, sy);
        break;
    }
}

// LB: resident blocks per SM the launch is built for (1: up to 128 registers a
// thread, the widest items without spills; 2: 64 registers, twice the warps to
// hide latency, for items of up to 4 columns).  The tuner picks.
template <int MODE, int LB>
__global__ void __launch_bounds__(kThreads, LB) k_batch(BatchParams B)
{
    __shared__ SharedM sh;
    __shared__ TeamShared ts;
    __shared__ int next;
    // this block's team entries, in the global schedule order
    for (int e = B.bptr[blockIdx.x]; e < B.bptr[blockIdx.x + 1]; e++) {
        const int2 ent = B.blist[e];
        if (!chk_in(CHK_ITEM, ent.x, B.n_all)) continue;
        const BatchItem &it = B.items[ent.x];
        const SolverParams P = item_params(it, B);
        const Ctx c = team_ctx(it, ent.y, it.team);
        const MultiParams M = it.M;
        if (threadIdx.x == 0) {
            ts.red = M.red;
            ts.ctr = it.ctr;
            ts.err = B.err;
            ts.limit_ns = B.timeout_ns;
            ts.arrive_ns = B.arrive_timeout_ns;
            ts.k = it.team;
            ts.r = ent.y;
            ts.epoch = 0u;
            ts.stall = B.stall_first;
        }
        __syncthreads();
        const unsigned long long t0 = mf_globaltimer();
        TeamSync sy{sh, ts};
        item_solve<MODE, (LB == 1 ? 8 : 4)>(P, M, it.nr, c, sh, sy);
        __syncthreads();
        if (ent.y == 0 && threadIdx.x == 0) {         // the item's start and end, for the report
            M.out[4 * it.nr + 3] = (double)t0;
            M.out[4 * it.nr + 4] = (double)mf_globaltimer();
        }
        if (*(volatile int *)B.err) return;      // a team wait gave up: the launch reports it
    }
    for (;;) {
        if (threadIdx.x == 0) next = (int)atomicAdd(B.head, 1u);
        __syncthreads();
        const int pos = next;
        __syncthreads();
        if (pos >= B.n_items) break;
        if (!chk_in(CHK_ITEM, B.order[pos], B.n_all)) continue;
        const BatchItem &it = B.items[B.order[pos]];
        const SolverParams P = item_params(it, B);
        const Ctx c = team_ctx(it, 0, 1);
        BlockSync sy{sh};
        const MultiParams M = it.M;
        const unsigned long long t0 = mf_globaltimer();
        item_solve<MODE, (LB == 1 ? 8 : 4)>(P, M, it.nr, c, sh, sy);
        __syncthreads();
        if (threadIdx.x == 0) {
            M.out[4 * it.nr + 3] = (double)t0;
            M.out[4 * it.nr + 4] = (double)mf_globaltimer();
        }
    }
}

// ------------------------------------------------------------ workspace
struct Workspace {
    int G;                 // grid blocks of the persistent kernel
    int lb;                // register-budget variant (blocks per SM it was built for)
    // every solver vector lives in one block, the FP64 CG set first, so one L2
    // access-policy window covers what a solve touches:
    //   p | q | r | x | s | t | rh | p32 | s32 | p16 | s16 | p8 | s8
    // (CG, FP64 / mixed: p..x; BiCGSTAB, FP64 / mixed: p..rh; parity mode: all)
    char *vecs;
    size_t cg_bytes, bicg_bytes, all_bytes;
    double *r, *p, *q, *rh, *s, *t, *x;
    float *p32, *s32, *mag_p, *mag_s;
    __half *p16, *s16;
    int8_t *p8, *s8;
    signed char *lab_p, *lab_s;
    double *red;
    unsigned int *bar;
    int *err;
    double *out;
    unsigned long long *counts;
    unsigned long long *phase_ns;
    int *hw_begin;
    int nhw;
    cudaEvent_t e0, e1;
    // several right-hand sides (k_solve_multi): interleaved vectors for NR columns
    int m_nr, m_G;
    double *m_vec;         // B | X | R | P | Q, each vec_len * NR
    float *m_mag;
    double *m_red, *m_out; // m_out: one result record per column group of a call (m_groups of them)
    int *m_err;            // one error word per column group
    int *m_hw_begin;
    int m_groups;          // column-group slots of m_out / m_err / m_ev
    cudaEvent_t *m_ev;     // two timing events per column group
};

template <typename T>
int dal(T **p, long long count)
{
    MF_CUDA_TRY(cudaMalloc((void **)p, (size_t)(count > 0 ? count : 1) * sizeof(T)));
    return MF_SUCCESS;
}

#define MF_TRY(expr)                        \
    do {                                    \
        int _rc = (expr);                   \
        if (_rc != MF_SUCCESS) return _rc;  \
    } while (0)

// count[0]: tiles exact in INT8 or FP16; count[1]: tiles within FP16's normal range
__global__ void k_count_exact(const unsigned char *caps, int n, unsigned long long *count)
{
    unsigned c = 0, h = 0, f = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        if (caps[t] & (MF_CAP_EXACT_I8 | MF_CAP_EXACT_F16)) c++;
        if (caps[t] & MF_CAP_FP16_OK) h++;
        if (caps[t] & MF_CAP_EXACT_F16) f++;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    h = __reduce_add_sync(0xffffffffu, h);
    f = __reduce_add_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
    if ((threadIdx.x & 31) == 0 && h) atomicAdd(count + 1, (unsigned long long)h);
    if ((threadIdx.x & 31) == 0 && f) atomicAdd(count + 2, (unsigned long long)f);
}

// Tiles exact in INT8 or FP16 (the lossless classes), tiles within FP16's
// normal range, and tiles exact in FP16, counted once per matrix through
// `scratch` (three unsigned long long of device memory).
int exact_tiles(mf_matrix_s *A, unsigned long long *scratch, cudaStream_t s)
{
    if (!A->n_exact_known) {
        unsigned long long h[3] = {0, 0, 0};
        MF_CUDA_TRY(cudaMemsetAsync(scratch, 0, sizeof(h), s));
        if (A->tilenum > 0) k_count_exact<<<256, 256, 0, s>>>(A->d_tile_caps, A->tilenum, scratch);
        MF_CUDA_TRY(cudaGetLastError());
        MF_CUDA_TRY(cudaMemcpyAsync(h, scratch, sizeof(h), cudaMemcpyDeviceToHost, s));
        MF_CUDA_TRY(cudaStreamSynchronize(s));
        A->n_exact = (long long)h[0];
        A->n_fp16_ok = (long long)h[1];
        A->n_exact_f16 = (long long)h[2];
        A->n_exact_known = 1;
    }
    return MF_SUCCESS;
}

// Lossless classes apply when asked for and enough tiles are exact in a narrower
// type (the same fraction that gates demotion by magnitude).
inline int lossless_on(int use_lossless, double min_fraction, long long n_exact, int tilenum)
{
    return (use_lossless && n_exact > 0 && (double)n_exact >= min_fraction * (double)tilenum) ? 1 : 0;
}

template <int METH>
const void *solve_kernel_m(int mode, int lb)
{
    if (lb == 2) {
        if (mode == MODE_FP64) return (const void *)k_solve<MODE_FP64, 2, METH>;
        if (mode == MODE_MIXED) return (const void *)k_solve<MODE_MIXED, 2, METH>;
        return (const void *)k_solve<MODE_PARITY, 2, METH>;
    }
    if (mode == MODE_FP64) return (const void *)k_solve<MODE_FP64, 1, METH>;
    if (mode == MODE_MIXED) return (const void *)k_solve<MODE_MIXED, 1, METH>;
    return (const void *)k_solve<MODE_PARITY, 1, METH>;
}

const void *solve_kernel(int mode, int lb, int method)
{
    return method == MF_METHOD_BICGSTAB ? solve_kernel_m<MF_METHOD_BICGSTAB>(mode, lb)
                                        : solve_kernel_m<MF_METHOD_CG>(mode, lb);
}

int ws_get(mf_matrix_s *A, int blocks_per_sm, Workspace **out, cudaStream_t s)
{
    // blocks_per_sm: 0 = default variant, 1 or 2 = that register-budget variant
    const int lb = (blocks_per_sm == 2) ? 2 : (blocks_per_sm == 1) ? 1 : kDefaultLB;
    int dev = 0;
    MF_CUDA_TRY(cudaGetDevice(&dev));
    int nsm = 0;
    MF_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    int coop = 0;
    MF_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) return MF_ERR_UNSUPPORTED;
    // one grid size for every precision mode, so the cached workspace is shared
    int occ = 1 << 20;
    for (int m = MODE_FP64; m <= MODE_PARITY; m++) {
        for (int meth = MF_METHOD_CG; meth <= MF_METHOD_BICGSTAB; meth++) {
            int o = 0;
            MF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, solve_kernel(m, lb, meth), kThreads, 0));
            occ = o < occ ? o : occ;
        }
    }
    if (occ < 1) return MF_ERR_UNSUPPORTED;
    if (occ > lb) occ = lb;
    int G = nsm * occ;
    // small systems: no more blocks than needed for one tile-row per half-warp
    const int need = (A->tilem + kWarps * 2 - 1) / (kWarps * 2);
    if (need < G) G = need > 0 ? need : 1;
    Workspace *w = (Workspace *)A->ws;
    if (w && w->G == G && w->lb == lb) {
        *out = w;
        return MF_SUCCESS;
    }
    if (w) mf_solver_free_ws(A);
    w = new Workspace();
    memset(w, 0, sizeof(*w));
    w->G = G;
    w->lb = lb;
    const long long L = A->vec_len;
    const long long S = std::max(A->tilem, A->tilen) + 1;
    {
        const size_t f = (size_t)L * sizeof(float), d = (size_t)L * sizeof(double), h = (size_t)L * sizeof(__half);
        w->cg_bytes = 4 * d;
        w->bicg_bytes = 7 * d;
        w->all_bytes = 7 * d + 2 * f + 2 * h + 2 * (size_t)L;
        MF_CUDA_TRY(cudaMalloc((void **)&w->vecs, w->all_bytes));
        char *c = w->vecs;
        w->p = (double *)c; c += d;
        w->q = (double *)c; c += d;
        w->r = (double *)c; c += d;
        w->x = (double *)c; c += d;
        w->s = (double *)c; c += d;
        w->t = (double *)c; c += d;
        w->rh = (double *)c; c += d;
        w->p32 = (float *)c; c += f;
        w->s32 = (float *)c; c += f;
        w->p16 = (__half *)c; c += h;
        w->s16 = (__half *)c; c += h;
        w->p8 = (int8_t *)c; c += L;
        w->s8 = (int8_t *)c;
    }
    MF_TRY(dal(&w->mag_p, S)); MF_TRY(dal(&w->mag_s, S));
    MF_TRY(dal(&w->lab_p, S)); MF_TRY(dal(&w->lab_s, S));
    MF_TRY(dal(&w->red, (long long)kRedKinds * G * kRedWidth));
    MF_TRY(dal(&w->bar, 1)); MF_TRY(dal(&w->err, 1)); MF_TRY(dal(&w->out, 16));
    MF_TRY(dal(&w->counts, 16));
    MF_TRY(dal(&w->phase_ns, 8));
    MF_TRY(exact_tiles(A, w->counts, s));    // counts: scratch before the first solve zeroes it
    w->nhw = G * kWarps * 2;
    MF_TRY(dal(&w->hw_begin, w->nhw + 1));
    MF_CUDA_TRY(cudaEventCreate(&w->e0));
    MF_CUDA_TRY(cudaEventCreate(&w->e1));
    k_partition<<<(w->nhw + 256) / 256, 256, 0, s>>>(A->d_row_cost, A->tilem, w->nhw, w->hw_begin);
    MF_CUDA_TRY(cudaGetLastError());
    A->ws = w;
    *out = w;
    return MF_SUCCESS;
}

void fill_params(SolverParams &P, mf_matrix_s *A, Workspace *w)
{
    memset(&P, 0, sizeof(P));
    P.n = A->n_rows;
    P.tilem = A->tilem;
    P.vec_len = A->vec_len;
    P.rowptr = A->d_rowptr;
    P.seg_ptr = A->d_seg_ptr;
    P.seg_hdr = A->d_seg_hdr;
    P.seg_rowlen = A->d_seg_rowlen;
    P.meta = A->d_meta;
    P.v64 = A->d_v64;
    P.v32 = A->d_v32;
    P.v16 = A->d_v16;
    P.v8 = A->d_v8;
    P.v8ref = A->d_v8ref;
    P.tile_col = A->d_tile_columnidx;
    P.seg_tile = A->d_seg_tile;
    P.tile_off = A->d_csr_offset;
    P.i8_scale = A->d_i8_scale;
    P.tile_caps = A->d_tile_caps;
    P.nseg = A->nseg;
    P.ntiles = A->tilenum;
    P.chk_xlen = A->vec_len;
    P.n_payload = A->slice_entries;
    if (w) {
        P.hw_begin = w->hw_begin;
        P.x = w->x; P.r = w->r; P.p = w->p; P.q = w->q; P.rh = w->rh; P.s = w->s; P.t = w->t;
        P.p32 = w->p32; P.s32 = w->s32; P.p16 = w->p16; P.s16 = w->s16; P.p8 = w->p8; P.s8 = w->s8;
        P.mag_p = w->mag_p; P.mag_s = w->mag_s; P.lab_p = w->lab_p; P.lab_s = w->lab_s;
        // CG in the FP64 / mixed modes multiplies r, not p: r's shadow takes p's slots
        P.mag_r = w->mag_p;
        P.red = w->red; P.bar = w->bar; P.err = w->err; P.out = w->out; P.counts = w->counts;
        P.phase_ns = w->phase_ns;
    }
}

// The first failed bounds check of the device since the last call (bounds-
// checked build): printed as site, index and limit, cleared, and returned as
// MF_ERR_CHECK.  Called after the entry point's own stream synchronisation.
// The normal build has no checks: MF_SUCCESS.
int chk_take()
{
#ifdef MF_CHECK
    unsigned long long h[3] = {0ull, 0ull, 0ull};
    if (cudaMemcpyFromSymbol(h, g_chk, sizeof(h)) != cudaSuccess) return MF_ERR_CUDA;
    if (h[0] == 0ull) return MF_SUCCESS;
    static const char *const kSite[CHK_NSITES] = {"",
                                                  "slice range",
                                                  "tile word / tile table",
                                                  "slice payload",
                                                  "gathered vector entry",
                                                  "row length",
                                                  "epilogue tile-row",
                                                  "batch queue entry"};
    fprintf(stderr, "millefeuille: bounds check failed: %s, index %lld, limit %lld\n",
            h[0] < (unsigned long long)CHK_NSITES ? kSite[h[0]] : "?", (long long)h[1], (long long)h[2]);
    const unsigned long long z[3] = {0ull, 0ull, 0ull};
    if (cudaMemcpyToSymbol(g_chk, z, sizeof(z)) != cudaSuccess) return MF_ERR_CUDA;
    return MF_ERR_CHECK;
#else
    return MF_SUCCESS;
#endif
}

// Persisting L2 access-policy window on a stream for the duration of a solve.
struct L2Window {
    bool active = false;
    size_t old_limit = 0;
    cudaStreamAttrValue old_attr;
    void set(cudaStream_t s, void *base, size_t bytes)
    {
        int dev = 0, max_persist = 0, max_win = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return;
        if (cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&max_win, cudaDevAttrMaxAccessPolicyWindowSize, dev) != cudaSuccess ||
            max_persist <= 0 || max_win <= 0) {
            cudaGetLastError();
            return;
        }
        if (cudaStreamGetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &old_attr) != cudaSuccess ||
            cudaDeviceGetLimit(&old_limit, cudaLimitPersistingL2CacheSize) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        const size_t win = bytes < (size_t)max_win ? bytes : (size_t)max_win;
        const size_t lim = win < (size_t)max_persist ? win : (size_t)max_persist;
        if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, lim) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        cudaStreamAttrValue a;
        memset(&a, 0, sizeof(a));
        a.accessPolicyWindow.base_ptr = base;
        a.accessPolicyWindow.num_bytes = win;
        a.accessPolicyWindow.hitRatio = (float)((double)lim / (double)win);
        a.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        a.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        if (cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &a) != cudaSuccess) {
            cudaGetLastError();
            cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, old_limit);
            return;
        }
        active = true;
    }
    void reset(cudaStream_t s)
    {
        if (!active) return;
        cudaStreamSetAttribute(s, cudaStreamAttributeAccessPolicyWindow, &old_attr);
        cudaCtxResetPersistingL2Cache();
        cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, old_limit);
        cudaGetLastError();
        active = false;
    }
};

}  // namespace

void mf_solver_free_ws(mf_matrix_s *A)
{
    Workspace *w = (Workspace *)A->ws;
    if (!w) return;
    void *ptrs[] = {w->vecs, w->mag_p, w->mag_s, w->lab_p, w->lab_s, w->red, w->bar, w->err, w->out, w->counts,
                    w->phase_ns, w->hw_begin, w->m_vec, w->m_mag, w->m_red, w->m_out, w->m_err, w->m_hw_begin};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (int k = 0; k < 2 * w->m_groups; k++) cudaEventDestroy(w->m_ev[k]);
    delete[] w->m_ev;
    cudaEventDestroy(w->e0);
    cudaEventDestroy(w->e1);
    delete w;
    A->ws = nullptr;
}

int mf_solver_run(mf_matrix_s *A, const double *d_b, double *d_x, const mf_options *opt, mf_report *rep,
                  cudaStream_t s)
{
    const int mode = opt->precision == MF_PREC_FP64 ? MODE_FP64
                     : opt->precision == MF_PREC_PARITY ? MODE_PARITY : MODE_MIXED;
    if (opt->method != MF_METHOD_CG && opt->method != MF_METHOD_BICGSTAB) return MF_ERR_INVALID;
    const auto t_begin = std::chrono::steady_clock::now();
    Workspace *w = nullptr;
    MF_TRY(ws_get(A, opt->blocks_per_sm, &w, s));
    const long long L = A->vec_len;
    const long long S = std::max(A->tilem, A->tilen) + 1;
    // zero the padded tails and the state the kernel reads before writing
    MF_CUDA_TRY(cudaMemsetAsync(w->x, 0, L * sizeof(double), s));
    if (opt->x0_given)
        MF_CUDA_TRY(cudaMemcpyAsync(w->x, d_x, (size_t)A->n_rows * sizeof(double), cudaMemcpyDeviceToDevice, s));
    MF_CUDA_TRY(cudaMemsetAsync(w->p, 0, L * sizeof(double), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->q, 0, L * sizeof(double), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->s, 0, L * sizeof(double), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->t, 0, L * sizeof(double), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->p32, 0, L * sizeof(float), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->s32, 0, L * sizeof(float), s));
    if (mode == MODE_PARITY) {
        MF_CUDA_TRY(cudaMemsetAsync(w->p16, 0, L * sizeof(__half), s));
        MF_CUDA_TRY(cudaMemsetAsync(w->s16, 0, L * sizeof(__half), s));
        MF_CUDA_TRY(cudaMemsetAsync(w->p8, 0, L, s));
        MF_CUDA_TRY(cudaMemsetAsync(w->s8, 0, L, s));
    }
    MF_CUDA_TRY(cudaMemsetAsync(w->mag_p, 0, S * sizeof(float), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->mag_s, 0, S * sizeof(float), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->lab_p, 0, S, s));
    MF_CUDA_TRY(cudaMemsetAsync(w->lab_s, 0, S, s));
    MF_CUDA_TRY(cudaMemsetAsync(w->bar, 0, sizeof(unsigned int), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->err, 0, sizeof(int), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->out, 0, 16 * sizeof(double), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->counts, 0, 16 * sizeof(unsigned long long), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->phase_ns, 0, 8 * sizeof(unsigned long long), s));
    SolverParams P;
    fill_params(P, A, w);
    P.b = d_b;
    P.method = opt->method;
    P.x0_given = opt->x0_given ? 1 : 0;
    P.max_iter = opt->max_iter;
    P.fixed_iters = opt->fixed_iters;
    P.replace_every = opt->replace_every;
    P.use_lossless = opt->use_lossless;
    P.lossless_any = lossless_on(opt->use_lossless, opt->demote_min_fraction, A->n_exact, A->tilenum);
    P.min_small = (float)(opt->demote_min_fraction * (double)A->tilem);
    P.min_demoted = (float)(opt->demote_min_fraction * (double)A->tilenum);
    P.relax_eta = (float)opt->relax_eta;
    P.relax_int8 = opt->relax_int8 ? 1 : 0;
    P.fp16_ok = A->n_fp16_ok == A->tilenum ? 1 : 0;
    // every tile exact in FP16: the lossless choice is the same for every tile and
    // every SpMV, so it is made here and the walk stays lookup-free (the per-slice
    // lookups with all tiles FP16 measured 37 % slower than the FP32 lean walk on
    // the 2048^2 Laplacian)
    if (opt->use_lossless && A->tilenum > 0 && A->n_exact_f16 == A->tilenum) {
        P.lean_f16 = 1;
        P.lossless_any = 0;
    }
    P.tol = opt->tol;
    P.demote16 = (float)opt->demote_fp16;
    P.demote8 = (float)opt->demote_int8;
    double to = opt->wait_timeout_s > 0 ? opt->wait_timeout_s : 10.0;
    P.timeout_ns = (unsigned long long)(to * 1e9);
    P.stall_first_barrier = opt->test_stall_barrier ? 1 : 0;
    if (opt->test_check_limit > 0) P.chk_xlen = (int)std::min<long long>(L, opt->test_check_limit & ~15LL);
    void *args[] = {&P};
    // Keep the iteration vectors in L2 while the matrix payload streams past
    // them: a persisting access-policy window over the vector block (best
    // effort; the previous stream attribute and context limit are restored).
    L2Window win;
    // (the FP64 / mixed modes never touch the narrow shadows: a smaller
    // persisting set-aside leaves more of L2 to the matrix stream -- measured
    // 3.5 % faster on the 128^3 system than a window that included p32)
    if (opt->l2_window)
        win.set(s, w->vecs, mode == MODE_PARITY ? w->all_bytes
                            : opt->method == MF_METHOD_BICGSTAB ? w->bicg_bytes : w->cg_bytes);
    const auto t_prepared = std::chrono::steady_clock::now();
    MF_CUDA_TRY(cudaEventRecord(w->e0, s));
    cudaError_t lerr = cudaLaunchCooperativeKernel(solve_kernel(mode, w->lb, opt->method), dim3(w->G), dim3(kThreads), args, 0, s);
    if (lerr != cudaSuccess) {
        win.reset(s);
        MF_CUDA_TRY(lerr);
    }
    MF_CUDA_TRY(cudaEventRecord(w->e1, s));
    double out[16];
    unsigned long long counts[16];
    int err = 0;
    MF_CUDA_TRY(cudaMemcpyAsync(out, w->out, sizeof(out), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaMemcpyAsync(counts, w->counts, sizeof(counts), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaMemcpyAsync(&err, w->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    unsigned long long phase[8];
    MF_CUDA_TRY(cudaMemcpyAsync(phase, w->phase_ns, sizeof(phase), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaMemcpyAsync(d_x, w->x, (size_t)A->n_rows * sizeof(double), cudaMemcpyDeviceToDevice, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    win.reset(s);
    const int chk = chk_take();
    if (chk) err = chk;
    const auto t_done = std::chrono::steady_clock::now();
    float ms = 0.f;
    MF_CUDA_TRY(cudaEventElapsedTime(&ms, w->e0, w->e1));
    if (rep) {
        memset(rep, 0, sizeof(*rep));
        rep->host_ms[1] = std::chrono::duration<double, std::milli>(t_prepared - t_begin).count();
        rep->host_ms[2] = std::chrono::duration<double, std::milli>(t_done - t_prepared).count();
        rep->iterations = (int)out[0];
        rep->converged = (int)out[1];
        rep->relres_true = out[2];
        rep->relres_rec = out[3];
        rep->residual = out[4];
        rep->replacements = (int)out[5];
        rep->status = err ? err : (int)out[6];
        rep->time_ms = ms;
        rep->grid_blocks = w->G;
        rep->threads_per_block = kThreads;
        for (int j = 0; j < 4; j++) rep->tile_uses[j] = (long long)counts[j];
        rep->tiles_skipped = (long long)counts[4];
        for (int j = 0; j < 4; j++) rep->nnz_uses[j] = (long long)counts[5 + j];
        if (mode == MODE_FP64) {
            // every tile of every SpMV phase runs in FP64: counted here, not in the kernel
            const long long nspmv = (long long)out[7];
            rep->tile_uses[0] = nspmv * A->tilenum;
            rep->nnz_uses[0] = nspmv * A->nnz;
        }
        for (int j = 0; j < 6; j++) rep->phase_ms[j] = (double)phase[j] * 1e-6;
    }
    if (err) return err;
    return (int)out[6];
}

// y = A x with every tile in one entry precision (MF_P64 .. MF_P8).
int mf_spmv_tiles_run(mf_matrix_s *A, const double *d_x, double *d_y, int tile_prec, cudaStream_t s,
                      double *elapsed_ms)
{
    if (tile_prec < MF_P64 || tile_prec > MF_P8) return MF_ERR_INVALID;
    // x is read through a padded copy so that column tiles past n_rows read zeros
    Workspace *w = nullptr;
    MF_TRY(ws_get(A, 0, &w, s));
    const long long L = A->vec_len;
    MF_CUDA_TRY(cudaMemsetAsync(w->x, 0, L * sizeof(double), s));
    MF_CUDA_TRY(cudaMemcpyAsync(w->x, d_x, (size_t)A->n_cols * sizeof(double), cudaMemcpyDeviceToDevice, s));
    SolverParams P;
    fill_params(P, A, w);
    int nsm = 0, dev = 0;
    MF_CUDA_TRY(cudaGetDevice(&dev));
    MF_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    // one wave: resident blocks x SMs, each half-warp a contiguous range of tile-rows
    const bool f64 = tile_prec == MF_P64;
    const void *kfn = f64 ? (const void *)k_spmv<MODE_FP64, 2> : (const void *)k_spmv<MODE_MIXED, 2>;
    int occ = 1;
    MF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, kThreads, 0));
    if (occ < 1) occ = 1;
    const int nhw_max = nsm * occ * kWarps * 2;
    int rows_per_hw = (A->tilem + nhw_max - 1) / nhw_max;
    if (rows_per_hw < 1) rows_per_hw = 1;
    const int nhw = (A->tilem + rows_per_hw - 1) / rows_per_hw;
    int blocks = (nhw + kWarps * 2 - 1) / (kWarps * 2);
    if (blocks < 1) blocks = 1;
    MF_CUDA_TRY(cudaEventRecord(w->e0, s));
    if (f64) k_spmv<MODE_FP64, 2><<<blocks, kThreads, 0, s>>>(P, MF_P64, d_y, rows_per_hw);
    else k_spmv<MODE_MIXED, 2><<<blocks, kThreads, 0, s>>>(P, tile_prec, d_y, rows_per_hw);
    MF_CUDA_TRY(cudaGetLastError());
    MF_CUDA_TRY(cudaEventRecord(w->e1, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    MF_TRY(chk_take());
    if (elapsed_ms) {
        float ms = 0.f;
        MF_CUDA_TRY(cudaEventElapsedTime(&ms, w->e0, w->e1));
        *elapsed_ms = ms;
    }
    return MF_SUCCESS;
}

int mf_spmv_run(mf_matrix_s *A, const double *d_x, double *d_y, int precision, cudaStream_t s, double *elapsed_ms)
{
    return mf_spmv_tiles_run(A, d_x, d_y, precision == MF_PREC_FP64 ? MF_P64 : MF_P32, s, elapsed_ms);
}

// The parity-mode labels the last solve left in the workspace (one per column
// segment), as d_vis codes.
int mf_solver_labels_run(mf_matrix_s *A, int *vis, int nseg)
{
    Workspace *w = (Workspace *)A->ws;
    if (!w || nseg < 0 || nseg > std::max(A->tilem, A->tilen)) return MF_ERR_INVALID;
    std::vector<signed char> h((size_t)nseg + 1);
    if (nseg > 0) MF_CUDA_TRY(cudaMemcpy(h.data(), w->lab_p, (size_t)nseg, cudaMemcpyDeviceToHost));
    for (int j = 0; j < nseg; j++) vis[j] = h[j];
    return MF_SUCCESS;
}

int mf_ref_labels_run(const double *d_pold, const double *d_pnew, int nseg, int *d_vis, cudaStream_t s)
{
    if (nseg <= 0) return MF_SUCCESS;
    const int threads = 256;
    const int segs_per_block = threads / 16;
    k_ref_labels<<<(nseg + segs_per_block - 1) / segs_per_block, threads, 0, s>>>(d_pold, d_pnew, nseg, d_vis);
    MF_CUDA_TRY(cudaGetLastError());
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    return MF_SUCCESS;
}

// ------------------------------------------------------------ tensor-core experiment (8 right-hand sides)
// Y = A X for 8 interleaved columns (row i's 8 values contiguous) with every
// tile's values stored in FP16, in two forms:
//  * CUDA cores (k_spmm_cc): the solver's arithmetic -- a half-warp per
//    tile-row, the FP16 value widened to FP64 against the FP64 row of X, 8
//    FP64 sums per row;
//  * tensor cores (k_spmm_tc): a warp per tile-row; each 16 x 16 tile of a
//    slice is densified in shared memory from the sparse payload (nothing
//    dense is read from HBM), X's 16 x 8 segment is rounded to FP16, and one
//    mma.sync.m16n8k16 per tile accumulates the 16 x 8 block in FP32.
// Both read the same slice payload; mf_debug_spmm times them side by side.
namespace {
__global__ void k_interleave(const double *B, int n, int L, int nrhs, int g, int NR, double *Bi);
__global__ void k_deinterleave(const double *Xi, int n, int nrhs, int g, int NR, double *X);

constexpr int kTcWarps = 4;                          // warps per block of k_spmm_tc
constexpr int kTcSmem = kTcWarps * MF_SEG_TILES * 256 * 2;   // dense FP16 tiles of one slice per warp

__global__ void __launch_bounds__(kThreads, 2) k_spmm_cc(SolverParams P, const double *X, double *Y)
{
    const int lane = threadIdx.x & 31, i = lane & 15;
    const unsigned hmask = 0xFFFFu << (16 * (lane >> 4));
    const int R = ((blockIdx.x * blockDim.x + threadIdx.x) >> 4);
    if (R >= P.tilem) return;
    double acc[8];
#pragma unroll
    for (int q = 0; q < 8; q++) acc[q] = 0.0;
    const int sb = P.seg_ptr[R], se = P.seg_ptr[R + 1];
    if (sb < se && (!chk_in(CHK_SLICE, sb, P.nseg) || !chk_in(CHK_SLICE, se - 1, P.nseg))) return;
    for (int s = sb; s < se; s++) {
        const int4 h = P.seg_hdr[s];
        const int xb = (load_tw(P, s, i) >> 8) * MF_BS;
        const int len = load_len(P, s, i, h);
        if (!chk_in(CHK_PAYLOAD, hdr_off(h) + (long long)hdr_kp(h) * MF_BS - 1, P.n_payload)) continue;
        for (int k0 = 0; k0 < hdr_kp(h); k0 += 8) {
            const long long cb = hdr_off(h) + (long long)(k0 >> 3) * 128;
            double v64[8];
            float v[8];
            load_chunk<MF_P16>(P, cb, i, len - k0, v64, v);
            const unsigned long long m8 = __ldcs((const unsigned long long *)(P.meta + cb) + i);
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const unsigned mm = (unsigned)(m8 >> (8 * j)) & 0xFFu;
                const int xi = __shfl_sync(hmask, xb, (int)(mm >> 4), 16) + (int)(mm & 15u);
                if (k0 + j < len && chk_in(CHK_X, xi, P.chk_xlen)) {
                    const double2 *xr = (const double2 *)(X + (long long)xi * 8);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const double2 d = xr[q];
                        acc[2 * q] = fma((double)v[j], d.x, acc[2 * q]);
                        acc[2 * q + 1] = fma((double)v[j], d.y, acc[2 * q + 1]);
                    }
                }
            }
        }
    }
    const int row = R * MF_BS + i;
    if (row < P.n) {
        double2 *yr = (double2 *)(Y + (long long)row * 8);
#pragma unroll
        for (int q = 0; q < 4; q++) yr[q] = make_double2(acc[2 * q], acc[2 * q + 1]);
    }
}

__device__ __forceinline__ unsigned pack_half2(double lo, double hi)
{
    return (unsigned)__half_as_ushort(__double2half(lo)) | ((unsigned)__half_as_ushort(__double2half(hi)) << 16);
}

__global__ void __launch_bounds__(kTcWarps * 32) k_spmm_tc(SolverParams P, const double *X, double *Y)
{
    extern __shared__ __align__(16) unsigned short tc_tiles[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int R = blockIdx.x * kTcWarps + w;
    if (R >= P.tilem) return;
    unsigned short *tiles = tc_tiles + w * MF_SEG_TILES * 256;   // [slot][row][col] FP16 bits
    const int g = lane >> 2, c = lane & 3;
    float d[4] = {0.f, 0.f, 0.f, 0.f};
    const int sb = P.seg_ptr[R], se = P.seg_ptr[R + 1];
    if (sb < se && (!chk_in(CHK_SLICE, sb, P.nseg) || !chk_in(CHK_SLICE, se - 1, P.nseg))) return;
    for (int s = sb; s < se; s++) {
        const int4 h = P.seg_hdr[s];
        const int nt = hdr_nt(h);
        if (!chk_in(CHK_PAYLOAD, hdr_off(h) + (long long)hdr_kp(h) * MF_BS - 1, P.n_payload)) continue;
        for (int e = lane; e < nt * 128; e += 32) ((unsigned *)tiles)[e] = 0u;
        __syncwarp();
        // lanes 0..15 scatter their row's entries into the dense tiles
        if (lane < 16) {
            const int len = load_len(P, s, lane, h);
            for (int k0 = 0; k0 < len; k0 += 8) {
                const long long cb = hdr_off(h) + (long long)(k0 >> 3) * 128;
                const uint4 u = __ldcs((const uint4 *)(P.v16 + cb) + lane);
                const unsigned long long m8 = __ldcs((const unsigned long long *)(P.meta + cb) + lane);
                const unsigned wv[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    if (k0 + j >= len) break;
                    const unsigned mm = (unsigned)(m8 >> (8 * j)) & 0xFFu;
                    if (!chk_in(CHK_TILE, (int)(mm >> 4), nt)) continue;
                    tiles[(mm >> 4) * 256 + lane * 16 + (mm & 15u)] =
                        (unsigned short)((wv[j >> 1] >> (16 * (j & 1))) & 0xFFFFu);
                }
            }
        }
        __syncwarp();
        const int tw = (lane < nt) ? load_tw(P, s, lane) : 0;
        for (int t = 0; t < nt; t++) {
            const int xb = (__shfl_sync(0xffffffffu, tw, t) >> 8) * MF_BS;
            const unsigned *T32 = (const unsigned *)(tiles + t * 256);
            // A (16 x 16, row-major) fragment of m16n8k16
            const unsigned a0 = T32[(g * 16 + 2 * c) >> 1], a1 = T32[((g + 8) * 16 + 2 * c) >> 1];
            const unsigned a2 = T32[(g * 16 + 2 * c + 8) >> 1], a3 = T32[((g + 8) * 16 + 2 * c + 8) >> 1];
            // B (16 x 8) fragment: X rows xb + k, column g, rounded to FP16
            const double *xr = X + (long long)xb * 8 + g;
            const unsigned b0 = pack_half2(xr[(2 * c) * 8], xr[(2 * c + 1) * 8]);
            const unsigned b1 = pack_half2(xr[(2 * c + 8) * 8], xr[(2 * c + 9) * 8]);
            asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
                         "{%8, %9}, {%0, %1, %2, %3};"
                         : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                         : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
        }
        __syncwarp();
    }
    const int r0 = R * MF_BS + g, r1 = r0 + 8;
    if (r0 < P.n) *(double2 *)(Y + (long long)r0 * 8 + 2 * c) = make_double2(d[0], d[1]);
    if (r1 < P.n) *(double2 *)(Y + (long long)r1 * 8 + 2 * c) = make_double2(d[2], d[3]);
}
}  // namespace

// Y = A X for 8 right-hand sides with FP16 stored values (the columns of X
// and Y one after another, n_cols / n_rows each); tensor_cores selects
// k_spmm_tc over k_spmm_cc.  elapsed_ms: the kernel alone.
int mf_spmm_run(mf_matrix_s *A, const double *d_X, double *d_Y, int tensor_cores, cudaStream_t s,
                double *elapsed_ms)
{
    Workspace *w = nullptr;
    MF_TRY(ws_get(A, 0, &w, s));
    const long long L = A->vec_len;
    double *Xi = nullptr, *Yi = nullptr;
    MF_TRY(dal(&Xi, L * 8));
    MF_TRY(dal(&Yi, L * 8));
    int rc = MF_SUCCESS;
    do {
        if (cudaMemsetAsync(Xi, 0, (size_t)L * 8 * sizeof(double), s) != cudaSuccess) { rc = MF_ERR_CUDA; break; }
        k_interleave<<<592, 256, 0, s>>>(d_X, A->n_cols, (int)L, 8, 0, 8, Xi);
        SolverParams P;
        fill_params(P, A, w);
        if (cudaEventRecord(w->e0, s) != cudaSuccess) { rc = MF_ERR_CUDA; break; }
        if (tensor_cores) {
            if (cudaFuncSetAttribute(k_spmm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem) != cudaSuccess) {
                rc = MF_ERR_CUDA;
                break;
            }
            k_spmm_tc<<<(A->tilem + kTcWarps - 1) / kTcWarps, kTcWarps * 32, kTcSmem, s>>>(P, Xi, Yi);
        } else {
            k_spmm_cc<<<(A->tilem * 16 + kThreads - 1) / kThreads, kThreads, 0, s>>>(P, Xi, Yi);
        }
        if (cudaGetLastError() != cudaSuccess || cudaEventRecord(w->e1, s) != cudaSuccess) { rc = MF_ERR_CUDA; break; }
        k_deinterleave<<<592, 256, 0, s>>>(Yi, A->n_rows, 8, 0, 8, d_Y);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) { rc = MF_ERR_CUDA; break; }
        rc = chk_take();
        float ms = 0.f;
        cudaEventElapsedTime(&ms, w->e0, w->e1);
        if (elapsed_ms) *elapsed_ms = ms;
    } while (0);
    cudaFree(Xi);
    cudaFree(Yi);
    return rc;
}

// ------------------------------------------------------------ allocation-free SpMV
// Scratch of mf_spmv_noalloc: the padded FP64 copy of x, as a file-scope device
// array (allocated with the module, one per device context), so the call
// itself allocates nothing.
static __device__ __align__(256) double g_noalloc_x[MF_SPMV_NOALLOC_MAX_LEN];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double *g_noalloc_x_addr[kMaxDevices];

// Device address of the scratch array on the current device, looked up once
// per device (cudaGetSymbolAddress; the first lookup may load the module) and
// kept while the library stays loaded.
int noalloc_scratch(int dev, double **x)
{
    if (dev < 0 || dev >= kMaxDevices) return MF_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_x_addr[dev]) {
        void *px = nullptr;
        MF_CUDA_TRY(cudaGetSymbolAddress(&px, g_noalloc_x));
        g_noalloc_x_addr[dev] = (double *)px;
    }
    *x = g_noalloc_x_addr[dev];
    return MF_SUCCESS;
}
}  // namespace

int mf_spmv_noalloc_run(mf_matrix_s *A, const double *d_x, double *d_y, int precision, cudaStream_t s)
{
    const long long L = A->vec_len;
    if (L > MF_SPMV_NOALLOC_MAX_LEN) return MF_ERR_UNSUPPORTED;
    int dev = 0;
    MF_CUDA_TRY(cudaGetDevice(&dev));
    if (dev != A->dev) return MF_ERR_INVALID;
    double *x = nullptr;
    MF_TRY(noalloc_scratch(dev, &x));
    // x, then zeros up to the padded length: every entry the kernel reads is written here
    MF_CUDA_TRY(cudaMemcpyAsync(x, d_x, (size_t)A->n_cols * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (L > A->n_cols)
        MF_CUDA_TRY(cudaMemsetAsync(x + A->n_cols, 0, (size_t)(L - A->n_cols) * sizeof(double), s));
    const int fpr = precision == MF_PREC_FP64 ? MF_P64 : MF_P32;
    SolverParams P;
    fill_params(P, A, nullptr);
    P.x = x;
    int nsm = 0;
    MF_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const void *kfn = fpr == MF_P64 ? (const void *)k_spmv<MODE_FP64, 2> : (const void *)k_spmv<MODE_MIXED, 2>;
    int occ = 1;
    MF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, kThreads, 0));
    if (occ < 1) occ = 1;
    const int nhw_max = nsm * occ * kWarps * 2;
    int rows_per_hw = (A->tilem + nhw_max - 1) / nhw_max;
    if (rows_per_hw < 1) rows_per_hw = 1;
    const int nhw = (A->tilem + rows_per_hw - 1) / rows_per_hw;
    int blocks = (nhw + kWarps * 2 - 1) / (kWarps * 2);
    if (blocks < 1) blocks = 1;
    if (fpr == MF_P64) k_spmv<MODE_FP64, 2><<<blocks, kThreads, 0, s>>>(P, MF_P64, d_y, rows_per_hw);
    else k_spmv<MODE_MIXED, 2><<<blocks, kThreads, 0, s>>>(P, MF_P32, d_y, rows_per_hw);
    MF_CUDA_TRY(cudaGetLastError());
    return MF_SUCCESS;
}

// ------------------------------------------------------------ several right-hand sides (host)
namespace {

// column block g of B (nrhs x n, one column after another) -> interleaved [row * NR + k]
__global__ void k_interleave(const double *B, int n, int L, int nrhs, int g, int NR, double *Bi)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)L * NR;
         t += (long long)gridDim.x * blockDim.x) {
        const int row = (int)(t / NR), k = (int)(t % NR), col = g * NR + k;
        Bi[t] = (row < n && col < nrhs) ? B[(long long)col * n + row] : 0.0;
    }
}
__global__ void k_deinterleave(const double *Xi, int n, int nrhs, int g, int NR, double *X)
{
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < (long long)n * NR;
         t += (long long)gridDim.x * blockDim.x) {
        const int row = (int)(t / NR), k = (int)(t % NR), col = g * NR + k;
        if (col < nrhs) X[(long long)col * n + row] = Xi[t];
    }
}

const void *multi_kernel(int mode, int nr)
{
    if (mode == MODE_FP64)
        return nr == 2 ? (const void *)k_solve_multi<MODE_FP64, 2>
               : nr == 4 ? (const void *)k_solve_multi<MODE_FP64, 4> : (const void *)k_solve_multi<MODE_FP64, 8>;
    return nr == 2 ? (const void *)k_solve_multi<MODE_MIXED, 2>
           : nr == 4 ? (const void *)k_solve_multi<MODE_MIXED, 4> : (const void *)k_solve_multi<MODE_MIXED, 8>;
}

// The multi-column workspace for NR columns (grid: one block of 512 threads per SM).
int ws_multi(mf_matrix_s *A, Workspace *w, int mode, int nr, cudaStream_t s)
{
    if (w->m_nr == nr && w->m_vec) return MF_SUCCESS;
    void *old[] = {w->m_vec, w->m_mag, w->m_red, w->m_hw_begin};
    for (void *p : old)
        if (p) cudaFree(p);
    w->m_vec = nullptr; w->m_mag = nullptr; w->m_red = nullptr;
    w->m_hw_begin = nullptr;
    w->m_nr = 0;
    int dev = 0, nsm = 0, occ = 0;
    MF_CUDA_TRY(cudaGetDevice(&dev));
    MF_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    for (int m = MODE_FP64; m <= MODE_MIXED; m++) {
        int o = 0;
        MF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, multi_kernel(m, nr), kThreads, 0));
        occ = (m == MODE_FP64 || o < occ) ? o : occ;
    }
    if (occ < 1) return MF_ERR_UNSUPPORTED;
    int G = nsm * (occ > 1 ? 1 : occ);
    const int need = (A->tilem + kWarps * 2 - 1) / (kWarps * 2);
    if (need < G) G = need > 0 ? need : 1;
    const long long L = A->vec_len, S = std::max(A->tilem, A->tilen) + 1;
    MF_TRY(dal(&w->m_vec, 5 * L * nr));
    MF_TRY(dal(&w->m_mag, S));
    MF_TRY(dal(&w->m_red, (long long)kRedKinds * G * kRedWidthM));
    MF_TRY(dal(&w->m_hw_begin, (long long)G * kWarps * 2 + 1));
    MF_CUDA_TRY(cudaMemsetAsync(w->m_vec, 0, (size_t)5 * L * nr * sizeof(double), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->m_mag, 0, (size_t)S * sizeof(float), s));
    const int nhw = G * kWarps * 2;
    k_partition<<<(nhw + 256) / 256, 256, 0, s>>>(A->d_row_cost, A->tilem, nhw, w->m_hw_begin);
    MF_CUDA_TRY(cudaGetLastError());
    w->m_G = G;
    w->m_nr = nr;
    return MF_SUCCESS;
}

constexpr int kOutM = 4 * kMaxNR + 8;    // doubles per column group's result record

// Result slots for `groups` column groups (grown, never shrunk).
int ws_multi_groups(Workspace *w, int groups)
{
    if (w->m_groups >= groups) return MF_SUCCESS;
    if (w->m_out) cudaFree(w->m_out);
    if (w->m_err) cudaFree(w->m_err);
    w->m_out = nullptr;
    w->m_err = nullptr;
    for (int k = 0; k < 2 * w->m_groups; k++) cudaEventDestroy(w->m_ev[k]);
    delete[] w->m_ev;
    w->m_ev = nullptr;
    w->m_groups = 0;
    MF_TRY(dal(&w->m_out, (long long)groups * kOutM));
    MF_TRY(dal(&w->m_err, groups));
    w->m_ev = new cudaEvent_t[2 * groups];
    for (int k = 0; k < 2 * groups; k++) MF_CUDA_TRY(cudaEventCreate(&w->m_ev[k]));
    w->m_groups = groups;
    return MF_SUCCESS;
}

}  // namespace

int mf_solver_multi_run(mf_matrix_s *A, int nrhs, const double *d_B, double *d_X, const mf_options *opt,
                        mf_report *reps, cudaStream_t s)
{
    if (opt->method != MF_METHOD_CG || opt->precision == MF_PREC_PARITY) return MF_ERR_UNSUPPORTED;
    const int mode = opt->precision == MF_PREC_FP64 ? MODE_FP64 : MODE_MIXED;
    Workspace *w = nullptr;
    MF_TRY(ws_get(A, opt->blocks_per_sm, &w, s));
    const int nr = nrhs >= 8 ? 8 : nrhs >= 4 ? 4 : 2;   // columns per launch
    MF_TRY(ws_multi(A, w, mode, nr, s));
    const long long L = A->vec_len;
    const int n = A->n_rows;
    SolverParams P;
    fill_params(P, A, w);
    P.hw_begin = w->m_hw_begin;
    P.method = MF_METHOD_CG;
    P.x0_given = opt->x0_given ? 1 : 0;
    P.max_iter = opt->max_iter;
    P.fixed_iters = opt->fixed_iters;
    P.replace_every = opt->replace_every;
    P.use_lossless = opt->use_lossless;
    P.lossless_any = lossless_on(opt->use_lossless, opt->demote_min_fraction, A->n_exact, A->tilenum);
    P.min_small = (float)(opt->demote_min_fraction * (double)A->tilem);
    P.min_demoted = (float)(opt->demote_min_fraction * (double)A->tilenum);
    P.tol = opt->tol;
    P.demote16 = (float)opt->demote_fp16;
    P.demote8 = (float)opt->demote_int8;
    const double to = opt->wait_timeout_s > 0 ? opt->wait_timeout_s : 10.0;
    P.timeout_ns = (unsigned long long)(to * 1e9);
    P.stall_first_barrier = opt->test_stall_barrier ? 1 : 0;
    MultiParams M;
    M.B = w->m_vec;
    M.X = w->m_vec + L * nr;
    M.R = w->m_vec + 2 * L * nr;
    M.Pv = w->m_vec + 3 * L * nr;
    M.Q = w->m_vec + 4 * L * nr;
    M.mag = w->m_mag;
    M.red = w->m_red;
    const int groups = (nrhs + nr - 1) / nr;
    MF_TRY(ws_multi_groups(w, groups));
    MF_CUDA_TRY(cudaMemsetAsync(w->m_out, 0, (size_t)groups * kOutM * sizeof(double), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->m_err, 0, (size_t)groups * sizeof(int), s));
    // every column group is enqueued back to back (the interleaved buffers are
    // reused in stream order); the host reads the results once, at the end
    for (int g = 0; g < groups; g++) {
        M.nr = std::min(nr, nrhs - g * nr);
        M.out = w->m_out + (size_t)g * kOutM;
        P.err = w->m_err + g;
        k_interleave<<<592, 256, 0, s>>>(d_B, n, (int)L, nrhs, g, nr, (double *)M.B);
        if (opt->x0_given) k_interleave<<<592, 256, 0, s>>>(d_X, n, (int)L, nrhs, g, nr, M.X);
        MF_CUDA_TRY(cudaGetLastError());
        MF_CUDA_TRY(cudaMemsetAsync(w->bar, 0, sizeof(unsigned int), s));
        void *args[] = {&P, &M};
        MF_CUDA_TRY(cudaEventRecord(w->m_ev[2 * g], s));
        MF_CUDA_TRY(cudaLaunchCooperativeKernel(multi_kernel(mode, nr), dim3(w->m_G), dim3(kThreads), args, 0, s));
        MF_CUDA_TRY(cudaEventRecord(w->m_ev[2 * g + 1], s));
        k_deinterleave<<<592, 256, 0, s>>>(M.X, n, nrhs, g, nr, d_X);
        MF_CUDA_TRY(cudaGetLastError());
    }
    std::vector<double> out((size_t)groups * kOutM);
    std::vector<int> err(groups);
    MF_CUDA_TRY(cudaMemcpyAsync(out.data(), w->m_out, out.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaMemcpyAsync(err.data(), w->m_err, err.size() * sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    int first_err = chk_take();
    for (int g = 0; g < groups; g++) {
        const double *o = out.data() + (size_t)g * kOutM;
        float ms = 0.f;
        MF_CUDA_TRY(cudaEventElapsedTime(&ms, w->m_ev[2 * g], w->m_ev[2 * g + 1]));
        const int status = err[g] ? err[g] : (int)o[4 * nr + 1];
        if (status != MF_SUCCESS && first_err == MF_SUCCESS) first_err = status;
        if (reps) {
            for (int k = 0; k < std::min(nr, nrhs - g * nr); k++) {
                mf_report *r = &reps[g * nr + k];
                memset(r, 0, sizeof(*r));
                r->status = status;
                r->iterations = (int)o[4 * k + 0];
                r->converged = (int)o[4 * k + 1];
                r->relres_true = o[4 * k + 2];
                r->relres_rec = o[4 * k + 3];
                r->time_ms = ms;
                r->replacements = (int)o[4 * nr + 2];
                r->grid_blocks = w->m_G;
                r->threads_per_block = kThreads;
            }
        }
    }
    return first_err;
}

// ------------------------------------------------------------ batched systems (host)
namespace {

struct BatchImpl {
    int dev = 0, cap = 8, lb = 1, nitems = 0, nsm = 0;
    int max_res[3] = {0, 0, 0};        // co-resident blocks of the k_batch<*, lb> launch, lb = 1, 2
    std::vector<mf_matrix_s *> sys;
    std::vector<int> nrhs;
    // items: system, first column, columns, interleave width, team size
    std::vector<int> it_sys, it_col0, it_ncol, it_nr, it_team;
    std::vector<BatchItem> h_items;
    BatchItem *d_items = nullptr;
    int *d_order = nullptr;            // queue items, largest estimated cost first
    int nqueue = 0;
    int grid = 1;                      // blocks of the launch
    int *d_bptr = nullptr;             // [grid + 1] team entries per block
    int2 *d_blist = nullptr;
    unsigned *d_ctl = nullptr;         // queue head | error word | one barrier counter per team item
    size_t ctl_bytes = 0;
    char *d_pool = nullptr;
    size_t pool_bytes = 0;
    std::vector<size_t> out_off;       // offset of each item's report words in the pool
    cudaStream_t own = nullptr;        // used when the caller passes the default stream
    cudaGraphExec_t graph = nullptr;
    std::vector<const void *> graph_key;
    int graph_mode = -1;
    cudaEvent_t e0 = nullptr, e1 = nullptr, e_in = nullptr;
    double last_ms = 0.0;

    void release_items()
    {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        graph_key.clear();
        void *p[] = {d_items, d_order, d_bptr, d_blist, d_ctl, d_pool};
        for (void *q : p)
            if (q) cudaFree(q);
        d_items = nullptr; d_order = nullptr; d_bptr = nullptr; d_blist = nullptr; d_ctl = nullptr;
        d_pool = nullptr;
    }
};

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr int kOutWords = 4 * kMaxNR + 8;

// Team sizes and the list schedule of team items.  fair = total cost / blocks;
// an item gets k = round(kTeamGrain x cost / fair) blocks, at most the launch and at most
// one block per kMinTeamRows tile-rows; k >= 2 makes it a team item.  Team
// items, largest first, go to the k blocks that are free first (ties: lower
// block), start = the latest of their free times, and those blocks are busy
// for cost / k.  Each block's list is sorted by (start, item).
void batch_schedule(const std::vector<double> &cost, const std::vector<int> &tilem, int grid, std::vector<int> &team,
                    std::vector<int> &bptr, std::vector<int2> &blist, std::vector<int> &queue)
{
    const int ni = (int)cost.size();
    double total = 0.0;
    for (double c : cost) total += c;
    const double fair = total / (double)std::max(1, grid);
    team.assign(ni, 1);
    std::vector<int> order(ni);
    for (int t = 0; t < ni; t++) order[t] = t;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<double> free_at(grid, 0.0);
    std::vector<std::vector<std::pair<double, int2>>> lists(grid);
    queue.clear();
    for (int t : order) {
        int k = 1;
        if (fair > 0.0 && grid > 1) {
            const double want = std::floor(kTeamGrain * cost[t] / fair + 0.5);
            k = (int)std::min<double>(want, (double)std::min(grid, std::max(1, tilem[t] / kMinTeamRows)));
            k = std::max(k, 1);
        }
        if (k < 2) {
            queue.push_back(t);
            continue;
        }
        team[t] = k;
        std::vector<int> blk(grid);
        for (int q = 0; q < grid; q++) blk[q] = q;
        std::stable_sort(blk.begin(), blk.end(), [&](int a, int b) { return free_at[a] < free_at[b]; });
        blk.resize(k);
        std::sort(blk.begin(), blk.end());
        double start = 0.0;
        for (int q : blk) start = std::max(start, free_at[q]);
        const double end = start + cost[t] / (double)k;
        for (int r = 0; r < k; r++) {
            free_at[blk[r]] = end;
            lists[blk[r]].push_back({start, make_int2(t, r)});
        }
    }
    bptr.assign(grid + 1, 0);
    blist.clear();
    for (int q = 0; q < grid; q++) {
        std::stable_sort(lists[q].begin(), lists[q].end(), [](const std::pair<double, int2> &a,
                                                             const std::pair<double, int2> &b) {
            return a.first < b.first || (a.first == b.first && a.second.x < b.second.x);
        });
        for (auto &e : lists[q]) blist.push_back(e.second);
        bptr[q + 1] = (int)blist.size();
    }
}

// Items for column cap `cap`: each system's right-hand sides in groups of <= cap,
// interleave width the next power of two (1, 2, 4, 8); team sizes and the
// schedule; all vectors in one pool.
int batch_build_items(BatchImpl &B, int cap, int lb, cudaStream_t s)
{
    B.release_items();
    B.cap = cap;
    B.lb = lb;
    B.it_sys.clear(); B.it_col0.clear(); B.it_ncol.clear(); B.it_nr.clear();
    for (int k = 0; k < (int)B.sys.size(); k++)
        for (int c0 = 0; c0 < B.nrhs[k]; c0 += cap) {
            const int g = std::min(cap, B.nrhs[k] - c0);
            B.it_sys.push_back(k);
            B.it_col0.push_back(c0);
            B.it_ncol.push_back(g);
            B.it_nr.push_back(mf_batch_width(g));
        }
    B.nitems = (int)B.it_sys.size();
    {
        // exact-tile counts of the systems (once per matrix)
        unsigned long long *scratch = nullptr;
        MF_CUDA_TRY(cudaMalloc((void **)&scratch, 3 * sizeof(*scratch)));
        int rc = MF_SUCCESS;
        for (mf_matrix_s *A : B.sys)
            if (rc == MF_SUCCESS) rc = exact_tiles(A, scratch, s);
        cudaFree(scratch);
        MF_TRY(rc);
    }
    std::vector<double> cost(B.nitems);
    std::vector<int> tilem(B.nitems);
    for (int t = 0; t < B.nitems; t++) {
        const mf_matrix_s *A = B.sys[B.it_sys[t]];
        cost[t] = mf_batch_item_cost(A->nnz, A->n_rows, B.it_nr[t]);
        tilem[t] = A->tilem;
    }
    // lb blocks per SM (all resident: the launch is cooperative)
    B.grid = std::max(1, std::min(B.max_res[lb], lb * B.nsm));
    std::vector<int> bptr, queue;
    std::vector<int2> blist;
    batch_schedule(cost, tilem, B.grid, B.it_team, bptr, blist, queue);
    if (blist.empty()) {
        // no team: one block per item at most
        B.grid = std::max(1, std::min(B.grid, B.nitems));
        bptr.assign(B.grid + 1, 0);
    }
    B.nqueue = (int)queue.size();
    // per item: B | X | R | P | Q (doubles), segment magnitudes,
    // report words, team partials
    std::vector<size_t> off(B.nitems), red_off(B.nitems, 0);
    size_t total = 0;
    B.out_off.assign(B.nitems, 0);
    for (int t = 0; t < B.nitems; t++) {
        const mf_matrix_s *A = B.sys[B.it_sys[t]];
        const size_t L = (size_t)A->vec_len, nr = (size_t)B.it_nr[t];
        off[t] = total;
        total += align256(5 * L * nr * sizeof(double)) + align256((size_t)(A->tilem + 1) * sizeof(float));
        B.out_off[t] = total;
        total += align256(kOutWords * sizeof(double));
        if (B.it_team[t] > 1) {
            red_off[t] = total;
            total += align256((size_t)kRedKinds * B.it_team[t] * kRedWidthM * sizeof(double));
        }
    }
    B.pool_bytes = total;
    MF_CUDA_TRY(cudaMalloc((void **)&B.d_pool, total > 0 ? total : 256));
    MF_CUDA_TRY(cudaMemsetAsync(B.d_pool, 0, total > 0 ? total : 256, s));
    int nteam = 0;
    std::vector<int> ctr_of(B.nitems, -1);
    for (int t = 0; t < B.nitems; t++)
        if (B.it_team[t] > 1) ctr_of[t] = nteam++;
    B.ctl_bytes = sizeof(unsigned) * (size_t)(2 + nteam);
    MF_CUDA_TRY(cudaMalloc((void **)&B.d_ctl, B.ctl_bytes));
    B.h_items.resize(B.nitems);
    for (int t = 0; t < B.nitems; t++) {
        const mf_matrix_s *A = B.sys[B.it_sys[t]];
        const size_t L = (size_t)A->vec_len, nr = (size_t)B.it_nr[t];
        BatchItem &it = B.h_items[t];
        memset(&it, 0, sizeof(it));
        it.seg_ptr = A->d_seg_ptr; it.seg_hdr = A->d_seg_hdr; it.seg_tile = A->d_seg_tile;
        it.seg_rowlen = A->d_seg_rowlen; it.meta = A->d_meta; it.v64 = A->d_v64; it.v32 = A->d_v32;
        it.v16 = A->d_v16; it.v8 = A->d_v8; it.i8_scale = A->d_i8_scale; it.row_cost = A->d_row_cost;
        it.n = A->n_rows; it.tilem = A->tilem; it.nr = (int)nr; it.team = B.it_team[t];
        it.n_exact = A->n_exact; it.tilenum = A->tilenum;
        it.nseg = A->nseg; it.vec_len = A->vec_len; it.n_payload = A->slice_entries;
        char *base = B.d_pool + off[t];
        double *v = (double *)base;
        it.M.B = v; it.M.X = v + L * nr; it.M.R = v + 2 * L * nr; it.M.Pv = v + 3 * L * nr; it.M.Q = v + 4 * L * nr;
        it.M.mag = (float *)(base + align256(5 * L * nr * sizeof(double)));
        it.M.red = it.team > 1 ? (double *)(B.d_pool + red_off[t]) : nullptr;
        it.M.out = (double *)(B.d_pool + B.out_off[t]);
        it.M.nr = B.it_ncol[t];
        it.ctr = it.team > 1 ? B.d_ctl + 2 + ctr_of[t] : nullptr;
    }
    MF_CUDA_TRY(cudaMalloc((void **)&B.d_items, sizeof(BatchItem) * (size_t)std::max(1, B.nitems)));
    MF_CUDA_TRY(cudaMalloc((void **)&B.d_order, sizeof(int) * (size_t)std::max(1, B.nqueue)));
    MF_CUDA_TRY(cudaMalloc((void **)&B.d_bptr, sizeof(int) * (size_t)(B.grid + 1)));
    MF_CUDA_TRY(cudaMalloc((void **)&B.d_blist, sizeof(int2) * (size_t)std::max<size_t>(1, blist.size())));
    if (B.nitems > 0)
        MF_CUDA_TRY(cudaMemcpyAsync(B.d_items, B.h_items.data(), sizeof(BatchItem) * B.nitems,
                                    cudaMemcpyHostToDevice, s));
    if (B.nqueue > 0)
        MF_CUDA_TRY(cudaMemcpyAsync(B.d_order, queue.data(), sizeof(int) * B.nqueue, cudaMemcpyHostToDevice, s));
    MF_CUDA_TRY(cudaMemcpyAsync(B.d_bptr, bptr.data(), sizeof(int) * (B.grid + 1), cudaMemcpyHostToDevice, s));
    if (!blist.empty())
        MF_CUDA_TRY(cudaMemcpyAsync(B.d_blist, blist.data(), sizeof(int2) * blist.size(), cudaMemcpyHostToDevice, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    return MF_SUCCESS;
}

// Enqueue one batched solve on s: interleave every item's columns, reset the
// queue head, error word and team counters, the cooperative persistent launch,
// de-interleave.  No host synchronisation.
int batch_enqueue(BatchImpl &B, const double *const *Bd, double *const *Xd, const BatchParams &bp0, int mode,
                  cudaStream_t s)
{
    for (int t = 0; t < B.nitems; t++) {
        const mf_matrix_s *A = B.sys[B.it_sys[t]];
        const int nr = B.it_nr[t], g = B.it_col0[t] / nr;
        k_interleave<<<148, 256, 0, s>>>(Bd[B.it_sys[t]], A->n_rows, A->vec_len, B.nrhs[B.it_sys[t]], g, nr,
                                          (double *)B.h_items[t].M.B);
        if (bp0.x0_given)          // the initial guesses: R = B - A X is formed in the launch
            k_interleave<<<148, 256, 0, s>>>(Xd[B.it_sys[t]], A->n_rows, A->vec_len, B.nrhs[B.it_sys[t]], g, nr,
                                              B.h_items[t].M.X);
    }
    MF_CUDA_TRY(cudaGetLastError());
    MF_CUDA_TRY(cudaMemsetAsync(B.d_ctl, 0, B.ctl_bytes, s));
    BatchParams bp = bp0;
    bp.items = B.d_items;
    bp.order = B.d_order;
    bp.n_items = B.nqueue;
    bp.n_all = B.nitems;
    bp.head = B.d_ctl;
    bp.err = (int *)(B.d_ctl + 1);
    bp.bptr = B.d_bptr;
    bp.blist = B.d_blist;
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(B.grid);
    cfg.blockDim = dim3(kThreads);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (B.lb == 2) {
        if (mode == MODE_FP64) MF_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_batch<MODE_FP64, 2>, bp));
        else MF_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_batch<MODE_MIXED, 2>, bp));
    } else {
        if (mode == MODE_FP64) MF_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_batch<MODE_FP64, 1>, bp));
        else MF_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_batch<MODE_MIXED, 1>, bp));
    }
    for (int t = 0; t < B.nitems; t++) {
        const mf_matrix_s *A = B.sys[B.it_sys[t]];
        const int nr = B.it_nr[t], g = B.it_col0[t] / nr;
        k_deinterleave<<<148, 256, 0, s>>>(B.h_items[t].M.X, A->n_rows, B.nrhs[B.it_sys[t]], g, nr,
                                            Xd[B.it_sys[t]]);
    }
    MF_CUDA_TRY(cudaGetLastError());
    return MF_SUCCESS;
}

}  // namespace

// The batch's team sizes and list schedule for given item costs (host only).
int mf_batch_schedule_impl(int nitems, const double *cost, const int *tilem, int grid, int *team, int *bptr,
                           int *blist, int *queue, int *nqueue)
{
    std::vector<double> c(cost, cost + nitems);
    std::vector<int> tm(tilem, tilem + nitems), tv, bp, q;
    std::vector<int2> bl;
    batch_schedule(c, tm, grid, tv, bp, bl, q);
    for (int t = 0; t < nitems; t++) team[t] = tv[t];
    for (int b = 0; b <= grid; b++) bptr[b] = bp[b];
    for (size_t e = 0; e < bl.size(); e++) {
        blist[2 * e] = bl[e].x;
        blist[2 * e + 1] = bl[e].y;
    }
    for (size_t k = 0; k < q.size(); k++) queue[k] = q[k];
    *nqueue = (int)q.size();
    return MF_SUCCESS;
}

struct mf_batch_s {
    BatchImpl impl;
};

int mf_batch_create_impl(mf_batch_s **out, int nsys, mf_matrix_s *const *systems, const int *nrhs, cudaStream_t s)
{
    mf_batch_s *b = new mf_batch_s();
    BatchImpl &B = b->impl;
    int rc = MF_SUCCESS;
    if (cudaGetDevice(&B.dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&B.nsm, cudaDevAttrMultiProcessorCount, B.dev) != cudaSuccess)
        rc = MF_ERR_CUDA;
    if (rc == MF_SUCCESS) {
        // co-resident blocks of the cooperative launch (both precisions, both register budgets)
        int o[4] = {0, 0, 0, 0};
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[0], k_batch<MODE_FP64, 1>, kThreads, 0) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[1], k_batch<MODE_MIXED, 1>, kThreads, 0) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[2], k_batch<MODE_FP64, 2>, kThreads, 0) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o[3], k_batch<MODE_MIXED, 2>, kThreads, 0) != cudaSuccess ||
            std::min(o[0], o[1]) < 1)
            rc = MF_ERR_CUDA;
        B.max_res[1] = std::min(o[0], o[1]) * B.nsm;
        B.max_res[2] = std::min(o[2], o[3]) * B.nsm;   // 0 if two blocks do not fit: never chosen
    }
    for (int k = 0; rc == MF_SUCCESS && k < nsys; k++) {
        if (!systems[k] || nrhs[k] < 1 || systems[k]->n_rows != systems[k]->n_cols || systems[k]->dev != B.dev) {
            rc = MF_ERR_INVALID;
            break;
        }
        B.sys.push_back(systems[k]);
        B.nrhs.push_back(nrhs[k]);
    }
    if (rc == MF_SUCCESS &&
        (cudaEventCreate(&B.e0) != cudaSuccess || cudaEventCreate(&B.e1) != cudaSuccess ||
         cudaEventCreateWithFlags(&B.e_in, cudaEventDisableTiming) != cudaSuccess ||
         cudaStreamCreateWithFlags(&B.own, cudaStreamNonBlocking) != cudaSuccess))
        rc = MF_ERR_CUDA;
    if (rc == MF_SUCCESS) rc = batch_build_items(B, 8, 1, s ? s : B.own);
    if (rc != MF_SUCCESS) {
        mf_batch_destroy_impl(b);
        return rc;
    }
    *out = b;
    return MF_SUCCESS;
}

void mf_batch_destroy_impl(mf_batch_s *b)
{
    if (!b) return;
    BatchImpl &B = b->impl;
    B.release_items();
    if (B.e0) cudaEventDestroy(B.e0);
    if (B.e1) cudaEventDestroy(B.e1);
    if (B.e_in) cudaEventDestroy(B.e_in);
    if (B.own) cudaStreamDestroy(B.own);
    delete b;
}

// Solve every system's right-hand sides.  Bd[k] / Xd[k]: device arrays of
// nrhs[k] x n_k doubles.  With use_graph the sequence is captured into a CUDA
// graph on first use and replayed while pointers, options and items stay the same.
int mf_batch_solve_impl(mf_batch_s *b, const double *const *Bd, double *const *Xd, const mf_options *opt,
                        mf_report *reps, int use_graph, cudaStream_t s)
{
    BatchImpl &B = b->impl;
    if (opt->method != MF_METHOD_CG || opt->precision == MF_PREC_PARITY) return MF_ERR_UNSUPPORTED;
    const int mode = opt->precision == MF_PREC_FP64 ? MODE_FP64 : MODE_MIXED;
    BatchParams bp;
    memset(&bp, 0, sizeof(bp));
    bp.max_iter = opt->max_iter;
    bp.fixed_iters = opt->fixed_iters;
    bp.replace_every = opt->replace_every;
    bp.use_lossless = opt->use_lossless;
    bp.tol = opt->tol;
    bp.min_fraction = opt->demote_min_fraction;
    bp.x0_given = opt->x0_given ? 1 : 0;
    bp.demote16 = (float)opt->demote_fp16;
    bp.demote8 = (float)opt->demote_int8;
    // team waits: within an item the members run in step (the normal bound);
    // arriving at an item may wait for members finishing earlier list entries
    const double to = opt->wait_timeout_s > 0 ? opt->wait_timeout_s : 10.0;
    bp.timeout_ns = (unsigned long long)(to * 1e9);
    bp.arrive_timeout_ns = (unsigned long long)(std::max(to * 30.0, 300.0) * 1e9);
    if (opt->test_stall_barrier) {
        // test hook: every team's first barrier waits for an arrival that never
        // comes and gives up after wait_timeout_s (MF_ERR_TIMEOUT, no fault)
        bp.stall_first = 1;
        bp.arrive_timeout_ns = bp.timeout_ns;
    }
    cudaStream_t run = s ? s : B.own;
    if (!s) {
        // the batch's own stream does not synchronise with the default stream on
        // its own: order it after the work already queued there (inputs, zeroing)
        MF_CUDA_TRY(cudaEventRecord(B.e_in, 0));
        MF_CUDA_TRY(cudaStreamWaitEvent(B.own, B.e_in, 0));
    }
    if (use_graph) {
        // the graph bakes in pointers, options and items: rebuilt when any changes
        std::vector<const void *> key;
        for (size_t k = 0; k < B.sys.size(); k++) {
            key.push_back(Bd[k]);
            key.push_back(Xd[k]);
        }
        const double opts[] = {opt->tol, (double)opt->max_iter, (double)opt->fixed_iters, (double)opt->replace_every,
                               opt->demote_fp16, opt->demote_int8, (double)opt->use_lossless, (double)B.cap,
                               (double)B.lb,
                               opt->wait_timeout_s, (double)opt->test_stall_barrier, opt->demote_min_fraction,
                               (double)opt->x0_given};
        for (double v : opts) {
            unsigned long long u;
            memcpy(&u, &v, sizeof(u));
            key.push_back((const void *)(uintptr_t)u);
        }
        if (!B.graph || key != B.graph_key || B.graph_mode != mode) {
            if (B.graph) cudaGraphExecDestroy(B.graph);
            B.graph = nullptr;
            cudaGraph_t g = nullptr;
            MF_CUDA_TRY(cudaStreamBeginCapture(run, cudaStreamCaptureModeThreadLocal));
            const int rc = batch_enqueue(B, Bd, Xd, bp, mode, run);
            const cudaError_t ce = cudaStreamEndCapture(run, &g);
            if (rc != MF_SUCCESS) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            MF_CUDA_TRY(ce);
            const cudaError_t ie = cudaGraphInstantiate(&B.graph, g, 0);
            cudaGraphDestroy(g);
            MF_CUDA_TRY(ie);
            B.graph_key = key;
            B.graph_mode = mode;
        }
        MF_CUDA_TRY(cudaEventRecord(B.e0, run));
        MF_CUDA_TRY(cudaGraphLaunch(B.graph, run));
        MF_CUDA_TRY(cudaEventRecord(B.e1, run));
    } else {
        MF_CUDA_TRY(cudaEventRecord(B.e0, run));
        MF_TRY(batch_enqueue(B, Bd, Xd, bp, mode, run));
        MF_CUDA_TRY(cudaEventRecord(B.e1, run));
    }
    std::vector<double> outs((size_t)B.nitems * kOutWords);
    for (int t = 0; t < B.nitems; t++)
        MF_CUDA_TRY(cudaMemcpyAsync(outs.data() + (size_t)t * kOutWords, B.d_pool + B.out_off[t],
                                    kOutWords * sizeof(double), cudaMemcpyDeviceToHost, run));
    int team_err = 0;
    MF_CUDA_TRY(cudaMemcpyAsync(&team_err, B.d_ctl + 1, sizeof(int), cudaMemcpyDeviceToHost, run));
    MF_CUDA_TRY(cudaStreamSynchronize(run));
    const int chk = chk_take();
    if (chk) team_err = chk;
    float ms = 0.f;
    MF_CUDA_TRY(cudaEventElapsedTime(&ms, B.e0, B.e1));
    B.last_ms = ms;
    int status = team_err;
    double t_first = 0.0;                  // the launch's first item start (globaltimer ns)
    for (int t = 0; t < B.nitems; t++) {
        const double ts = outs[(size_t)t * kOutWords + 4 * B.it_nr[t] + 3];
        if (ts > 0.0 && (t_first == 0.0 || ts < t_first)) t_first = ts;
    }
    std::vector<int> first(B.sys.size() + 1, 0);
    for (size_t k = 0; k < B.sys.size(); k++) first[k + 1] = first[k] + B.nrhs[k];
    for (int t = 0; t < B.nitems; t++) {
        const double *o = outs.data() + (size_t)t * kOutWords;
        const int nr = B.it_nr[t];
        if ((int)o[4 * nr + 1] != MF_SUCCESS && status == MF_SUCCESS) status = (int)o[4 * nr + 1];
        if (!reps) continue;
        for (int c = 0; c < B.it_ncol[t]; c++) {
            mf_report *r = &reps[first[B.it_sys[t]] + B.it_col0[t] + c];
            memset(r, 0, sizeof(*r));
            r->iterations = (int)o[4 * c + 0];
            r->converged = (int)o[4 * c + 1];
            r->relres_true = o[4 * c + 2];
            r->relres_rec = o[4 * c + 3];
            r->status = team_err ? team_err : (int)o[4 * nr + 1];
            r->replacements = (int)o[4 * nr + 2];
            r->time_ms = ms;
            r->phase_ms[0] = o[4 * nr + 3] > 0.0 ? (o[4 * nr + 3] - t_first) * 1e-6 : 0.0;
            r->phase_ms[1] = o[4 * nr + 4] > 0.0 ? (o[4 * nr + 4] - t_first) * 1e-6 : 0.0;
            r->phase_ms[2] = (double)B.it_team[t];
            r->grid_blocks = B.grid;
            r->threads_per_block = kThreads;
        }
    }
    return status;
}

// Right-hand sides per work item chosen by timing: each candidate cap runs
// `iters` fixed iterations of the real batch with all-ones right-hand sides.
// A given (columns per item, blocks per SM), e.g. what mf_batch_tune chose for
// a batch of the same systems' shapes: the same item build, no timing runs.
int mf_batch_configure_impl(mf_batch_s *b, int cap, int lb, cudaStream_t s)
{
    BatchImpl &B = b->impl;
    if (cap != 1 && cap != 2 && cap != 4 && cap != 8) return MF_ERR_INVALID;
    // two blocks per SM only for items of up to 4 columns, as the tuner's candidates
    if (lb != 1 && !(lb == 2 && cap <= 4 && B.max_res[2] >= 1)) return MF_ERR_INVALID;
    return batch_build_items(B, cap, lb, s ? s : B.own);
}

void mf_batch_config_impl(const mf_batch_s *b, int *cap, int *lb)
{
    if (cap) *cap = b->impl.cap;
    if (lb) *lb = b->impl.lb;
}

int mf_batch_tune_impl(mf_batch_s *b, int precision, int iters, int *chosen, cudaStream_t s)
{
    BatchImpl &B = b->impl;
    cudaStream_t run = s ? s : B.own;
    std::vector<double *> bufB(B.sys.size(), nullptr), bufX(B.sys.size(), nullptr);
    int rc = MF_SUCCESS;
    for (size_t k = 0; k < B.sys.size() && rc == MF_SUCCESS; k++) {
        const size_t e = (size_t)B.nrhs[k] * B.sys[k]->n_rows;
        if (cudaMalloc((void **)&bufB[k], 2 * e * sizeof(double) + 16) != cudaSuccess) {
            rc = MF_ERR_NOMEM;
            break;
        }
        bufX[k] = bufB[k] + e;
        std::vector<double> ones(e, 1.0);
        if (cudaMemcpy(bufB[k], ones.data(), e * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = MF_ERR_CUDA;
    }
    mf_options o;
    mf_options_default(&o);
    o.precision = precision;
    o.fixed_iters = 1;
    o.max_iter = iters;
    o.replace_every = 0;
    // (columns per item, blocks per SM): two blocks per SM only for items of up
    // to 4 columns (8-column items need the 128-register budget)
    const int cand[][2] = {{8, 1}, {4, 1}, {2, 1}, {4, 2}, {2, 2}};
    int best = 8, best_lb = 1;
    double best_ms = 1e300;
    for (const auto &cl : cand) {
        if (rc != MF_SUCCESS) break;
        if (cl[1] == 2 && B.max_res[2] < 1) continue;
        if ((rc = batch_build_items(B, cl[0], cl[1], run)) != MF_SUCCESS) break;
        // the first run warms up; the faster of the next two counts (one timed
        // run of 20 iterations picked two blocks per SM where one was 7 %
        // faster over the whole 512-system batch)
        double ms = 1e300;
        for (int rep = 0; rep < 3 && rc == MF_SUCCESS; rep++) {
            rc = mf_batch_solve_impl(b, bufB.data(), bufX.data(), &o, nullptr, 0, run);
            if (rep > 0) ms = std::min(ms, B.last_ms);
        }
        // Two blocks per SM (64 registers, the multi-column walk spills) win the
        // short probe, where every item is active, but lose a full solve, whose
        // end is a tail of a few long items run at per-block speed: on the
        // 512-system batch the probe measured 315 ms (4 columns, 2 blocks)
        // against 344 ms (4 columns, 1 block), and the whole solve 13.2 s
        // against 11.2 s.  They count 15 % slower than measured.
        const double score = cl[1] == 2 ? 1.15 * ms : ms;
        if (rc == MF_SUCCESS && score < best_ms) {
            best_ms = score;
            best = cl[0];
            best_lb = cl[1];
        }
    }
    for (size_t k = 0; k < B.sys.size(); k++)
        if (bufB[k]) cudaFree(bufB[k]);
    if (rc == MF_SUCCESS) rc = batch_build_items(B, best, best_lb, run);
    if (chosen) *chosen = best;
    return rc;
}
