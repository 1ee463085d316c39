// tile_build.cu -- GPU csr2block, precision encoder and solver-slice builder.
//
// Produces, on the device, the reference tile layout bit-exact to Tile_create
// (csr2block.h:267-422), the offsets of blockspmv_cpu (blockspmv_cpu.h:35-111),
// the nonempty-row lists of cg_solve_inc (main-cg-mixed.cu:2447-2514), the
// encoder arrays (main-cg-mixed.cu:2333-2350) and this library's solver slices.
//
// One warp per tile-row.  The distinct column tiles of a tile-row are found
// with a bitmap over the tile-row's column-tile span (in shared memory, or in
// a global scratch slice when the span is too wide), ranked with popcounts,
// so the tile order is ascending as in convert_step2 (csr2block.h:89-102).
// Entries are then ranked inside their tile in CSR order with __match_any_sync
// (the order convert_step4 appends them in, csr2block.h:204-219).
#include "mf_internal.cuh"

#include <algorithm>
#include <chrono>
#include <vector>

namespace {

constexpr int kWarps = 8;           // warps per block in the per-tile-row kernels
constexpr int kThreads = kWarps * 32;

__device__ __forceinline__ int tile_row_end(int R, int tilem, int rowA)
{
    return (R == tilem - 1) ? rowA : (R + 1) * MF_BS;
}

// ---- K0: column-tile span per tile-row, and the maxima the host needs ----
__global__ void k_span(const int *__restrict__ rowptr, const int *__restrict__ colidx, int tilem, int rowA,
                       int colA, int *__restrict__ span_base, int *__restrict__ maxes, int *__restrict__ err)
{
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int R = warp; R < tilem; R += nwarps) {
        const int a = rowptr[R * MF_BS], b = rowptr[tile_row_end(R, tilem, rowA)];
        int jmin = INT_MAX, jmax = -1;
        bool bad = (b < a);
        for (int j = a + lane; j < b; j += 32) {
            int c = colidx[j];
            if (c < 0 || c >= colA) { bad = true; continue; }
            int jc = c >> 4;
            jmin = min(jmin, jc);
            jmax = max(jmax, jc);
        }
        for (int o = 16; o; o >>= 1) {
            jmin = min(jmin, __shfl_xor_sync(0xffffffffu, jmin, o));
            jmax = max(jmax, __shfl_xor_sync(0xffffffffu, jmax, o));
        }
        bad = __any_sync(0xffffffffu, bad);
        if (lane == 0) {
            if (bad) atomicExch(err, MF_ERR_INVALID);
            int words = (jmax < 0) ? 0 : (jmax >> 5) - (jmin >> 5) + 1;
            span_base[R] = (jmax < 0) ? 0 : (jmin >> 5);
            atomicMax(&maxes[0], words);
            atomicMax(&maxes[1], b - a);
        }
    }
}

// scratch layout per warp (32-bit words): bitmap[span], prefix[span], cnt[max_tiles]
struct Scratch {
    unsigned int *bm;
    int *pre;
    int *cnt;
};

__device__ __forceinline__ Scratch warp_scratch(unsigned int *smem, unsigned int *gscratch, int words_per_warp,
                                                int span, int global_mode)
{
    const int wib = threadIdx.x >> 5;
    const long long gw = (long long)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    unsigned int *base = global_mode ? gscratch + gw * (long long)words_per_warp : smem + (long long)wib * words_per_warp;
    Scratch s;
    s.bm = base;
    s.pre = (int *)(base + span);
    s.cnt = (int *)(base + 2 * span);
    return s;
}

// Build the tile-row bitmap; returns the number of distinct tiles.
__device__ int build_bitmap(const Scratch &S, const int *__restrict__ colidx, int a, int b, int base_word,
                            int words, int lane)
{
    for (int w = lane; w < words; w += 32) S.bm[w] = 0u;
    __syncwarp();
    for (int j = a + lane; j < b; j += 32) {
        int jc = colidx[j] >> 4;
        atomicOr(&S.bm[(jc >> 5) - base_word], 1u << (jc & 31));
    }
    __syncwarp();
    int cnt = 0;
    for (int w = lane; w < words; w += 32) cnt += __popc(S.bm[w]);
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    return cnt;
}

// ---- K1: distinct tiles per tile-row ----
__global__ void k_count_tiles(const int *__restrict__ rowptr, const int *__restrict__ colidx, int tilem, int rowA,
                              const int *__restrict__ span_base, int span, int words_per_warp, int global_mode,
                              unsigned int *gscratch, int *__restrict__ ntiles)
{
    extern __shared__ unsigned int smem[];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    Scratch S = warp_scratch(smem, gscratch, words_per_warp, span, global_mode);
    for (int R = warp; R < tilem; R += nwarps) {
        const int a = rowptr[R * MF_BS], b = rowptr[tile_row_end(R, tilem, rowA)];
        const int base_word = span_base[R];
        int words = 0;
        if (b > a) {
            int jmax_word = base_word;   // recompute the span of this tile-row
            int jm = -1;
            for (int j = a + lane; j < b; j += 32) jm = max(jm, colidx[j] >> 4);
            for (int o = 16; o; o >>= 1) jm = max(jm, __shfl_xor_sync(0xffffffffu, jm, o));
            jmax_word = jm >> 5;
            words = jmax_word - base_word + 1;
        }
        int c = (words > 0) ? build_bitmap(S, colidx, a, b, base_word, words, lane) : 0;
        if (lane == 0) ntiles[R] = c;
        __syncwarp();
    }
}

// ---- K2: tile columns, payload offsets, scatter, uint8 row starts ----
__global__ void k_fill_tiles(const int *__restrict__ rowptr, const int *__restrict__ colidx,
                             const double *__restrict__ val, const float *__restrict__ val_low, int tilem,
                             int rowA, const int *__restrict__ span_base, int span, int words_per_warp,
                             int global_mode, unsigned int *gscratch, const int *__restrict__ tile_ptr,
                             int *__restrict__ tile_columnidx, int *__restrict__ csr_offset,
                             int *__restrict__ csrptr_offset, double *__restrict__ tval,
                             float *__restrict__ tval_low, unsigned char *__restrict__ tcol,
                             unsigned char *__restrict__ tptr, int *__restrict__ err)
{
    extern __shared__ unsigned int smem[];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    Scratch S = warp_scratch(smem, gscratch, words_per_warp, span, global_mode);
    const int nz0 = rowptr[0];
    for (int R = warp; R < tilem; R += nwarps) {
        const int rs = R * MF_BS, re = tile_row_end(R, tilem, rowA);
        const int rowlen = re - rs;
        const int a = rowptr[rs], b = rowptr[re];
        const int t0 = tile_ptr[R], nt = tile_ptr[R + 1] - t0;
        // csrptr_offset: exclusive scan of tile-row heights over tiles (csr2block.h:146,347)
        for (int s = lane; s < nt; s += 32) csrptr_offset[t0 + s] = t0 * MF_BS + s * rowlen;
        if (R == tilem - 1 && lane == 0) csrptr_offset[t0 + nt] = t0 * MF_BS + nt * rowlen;
        if (nt == 0) {
            if (R == tilem - 1 && lane == 0) csr_offset[t0] = b - nz0;
            continue;
        }
        const int base_word = span_base[R];
        int jm = -1;
        for (int j = a + lane; j < b; j += 32) jm = max(jm, colidx[j] >> 4);
        for (int o = 16; o; o >>= 1) jm = max(jm, __shfl_xor_sync(0xffffffffu, jm, o));
        const int words = (jm >> 5) - base_word + 1;
        build_bitmap(S, colidx, a, b, base_word, words, lane);
        // exclusive popcount prefix over the bitmap words
        int carry = 0;
        for (int w0 = 0; w0 < words; w0 += 32) {
            int w = w0 + lane;
            int c = (w < words) ? __popc(S.bm[w]) : 0;
            int incl = c;
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            if (w < words) S.pre[w] = carry + incl - c;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        __syncwarp();
        // tile_columnidx, ascending
        for (int w = lane; w < words; w += 32) {
            unsigned int m = S.bm[w];
            int r = S.pre[w];
            while (m) {
                int bit = __ffs(m) - 1;
                m &= m - 1u;
                tile_columnidx[t0 + r] = (base_word + w) * 32 + bit;
                r++;
            }
        }
        // pass 1: entries per tile
        for (int s = lane; s < nt; s += 32) S.cnt[s] = 0;
        __syncwarp();
        for (int j = a + lane; j < b; j += 32) {
            int jc = colidx[j] >> 4;
            int w = (jc >> 5) - base_word, bit = jc & 31;
            int slot = S.pre[w] + __popc(S.bm[w] & ((1u << bit) - 1u));
            atomicAdd(&S.cnt[slot], 1);
        }
        __syncwarp();
        // payload offsets: tile-row payload starts at rowptr[rs] (csr_offset scan)
        int run = a - nz0;
        for (int s0 = 0; s0 < nt; s0 += 32) {
            int s = s0 + lane;
            int c = (s < nt) ? S.cnt[s] : 0;
            int incl = c;
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            if (s < nt) {
                csr_offset[t0 + s] = run + incl - c;
                if (c > 256) atomicExch(err, MF_ERR_UNSUPPORTED);   // duplicate columns overflow a tile
            }
            run += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (R == tilem - 1 && lane == 0) csr_offset[t0 + nt] = run;
        __syncwarp();
        for (int s = lane; s < nt; s += 32) S.cnt[s] = 0;
        __syncwarp();
        // pass 2: row by row in CSR order
        for (int ri = 0; ri < rowlen; ri++) {
            for (int s = lane; s < nt; s += 32) {
                int c = S.cnt[s];
                if (c > 255) atomicExch(err, MF_ERR_UNSUPPORTED);
                // csrptr_offset[t0 + s] = t0 * 16 + s * rowlen (only the last tile-row is short)
                tptr[(long long)t0 * MF_BS + (long long)s * rowlen + ri] = (unsigned char)c;
            }
            __syncwarp();
            const int ja = rowptr[rs + ri], jb = rowptr[rs + ri + 1];
            for (int j0 = ja; j0 < jb; j0 += 32) {
                int j = j0 + lane;
                bool act = j < jb;
                unsigned amask = __ballot_sync(0xffffffffu, act);
                int slot = 0, c = 0;
                if (act) {
                    c = colidx[j];
                    int jc = c >> 4;
                    int w = (jc >> 5) - base_word, bit = jc & 31;
                    slot = S.pre[w] + __popc(S.bm[w] & ((1u << bit) - 1u));
                }
                unsigned grp = __match_any_sync(0xffffffffu, act ? slot : -1);
                if (act) {
                    int rank = __popc(grp & lt_mask);
                    int pos = S.cnt[slot] + rank;
                    int o = csr_offset[t0 + slot] + pos;
                    tval[o] = val[j];
                    tval_low[o] = val_low ? val_low[j] : (float)val[j];
                    tcol[o] = (unsigned char)(c & 15);
                }
                __syncwarp();
                if (act && (grp & lt_mask) == 0) S.cnt[slot] += __popc(grp);
                __syncwarp();
                (void)amask;
            }
        }
        __syncwarp();
    }
}

// ---- rowlists: nonempty rows per tile (main-cg-mixed.cu:2455-2514) ----
__device__ __forceinline__ int tile_row_stop(const unsigned char *ptr, int cc, int ri, int rowlen, int nnzt)
{
    return (ri == rowlen - 1) ? nnzt : (int)ptr[cc + ri + 1];
}

// Row start as the reference stores it.  exclusive_scan_char returns early for
// length 1 (utils.h:52-53), so a one-row tile-row keeps its row count as the
// "start" (csr2block.h:237,252).  The device ptr array holds the true start 0;
// the reference value is restated here and in the exported copy.
__device__ __forceinline__ int ref_row_start(const unsigned char *ptr, int cc, int ri, int rowlen, int nnzt)
{
    return (rowlen == 1) ? (int)(unsigned char)nnzt : (int)ptr[cc + ri];
}

__global__ void k_rowlist_count(const int *__restrict__ tile_ptr, const int *__restrict__ csr_offset,
                                const int *__restrict__ csrptr_offset, const unsigned char *__restrict__ tptr,
                                int tilem, int rowA, int *__restrict__ nzr, int *__restrict__ tile_rowidx,
                                int *__restrict__ block_signal)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int R = warp; R < tilem; R += nwarps) {
        const int rowlen = (R == tilem - 1) ? rowA - R * MF_BS : MF_BS;
        const int t0 = tile_ptr[R], t1 = tile_ptr[R + 1];
        if (lane == 0) block_signal[R] = t1 - t0;
        for (int t = t0 + lane; t < t1; t += 32) {
            tile_rowidx[t] = R;
            const int cc = csrptr_offset[t];
            const int nnzt = csr_offset[t + 1] - csr_offset[t];
            int cnt = 0;
            for (int ri = 0; ri < rowlen; ri++)
                if (tile_row_stop(tptr, cc, ri, rowlen, nnzt) != ref_row_start(tptr, cc, ri, rowlen, nnzt)) cnt++;
            nzr[t] = cnt + 1;
        }
    }
}

__global__ void k_rowlist_fill(const int *__restrict__ tile_ptr, const int *__restrict__ csr_offset,
                               const int *__restrict__ csrptr_offset, const unsigned char *__restrict__ tptr,
                               int tilem, int rowA, const int *__restrict__ nzr_scan,
                               unsigned char *__restrict__ rowid, unsigned char *__restrict__ cptr)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int R = warp; R < tilem; R += nwarps) {
        const int rowlen = (R == tilem - 1) ? rowA - R * MF_BS : MF_BS;
        for (int t = tile_ptr[R] + lane; t < tile_ptr[R + 1]; t += 32) {
            const int cc = csrptr_offset[t];
            const int nnzt = csr_offset[t + 1] - csr_offset[t];
            int base = nzr_scan[t], fl = 0;
            for (int ri = 0; ri < rowlen; ri++) {
                int stop = tile_row_stop(tptr, cc, ri, rowlen, nnzt);
                if (ri == 0) { rowid[base + fl] = 0; cptr[base + fl] = 0; fl++; }
                if (stop != ref_row_start(tptr, cc, ri, rowlen, nnzt)) {
                    rowid[base + fl] = (unsigned char)ri;
                    cptr[base + fl] = (unsigned char)stop;
                    fl++;
                }
            }
        }
    }
}

// ---- row-block split of blockspmv_cpu (blockspmv_cpu.h:35-83), PREFETCH_SMEM_TH = 4 ----
__global__ void k_rowblk_count(const int *__restrict__ tile_ptr, int tilem, int *__restrict__ cnt)
{
    int R = blockIdx.x * blockDim.x + threadIdx.x;
    if (R >= tilem) return;
    int nb = tile_ptr[R + 1] - tile_ptr[R];
    cnt[R] = (nb <= 4) ? 1 : (nb + 3) / 4;
}

__global__ void k_rowblk_fill(const int *__restrict__ tile_ptr, int tilem, const int *__restrict__ off,
                              unsigned int *__restrict__ idx, int *__restrict__ cs, int *__restrict__ ce)
{
    int R = blockIdx.x * blockDim.x + threadIdx.x;
    if (R >= tilem) return;
    int nb = tile_ptr[R + 1] - tile_ptr[R];
    int o = off[R];
    if (nb <= 4) {
        idx[o] = (unsigned)R; cs[o] = 0; ce[o] = 0;
        return;
    }
    int num = (nb + 3) / 4;
    int len = (nb + num - 1) / num;
    for (int i = 0; i < num; i++) {
        idx[o + i] = (unsigned)R | 0x80000000u;
        cs[o + i] = tile_ptr[R] + i * len;
        ce[o + i] = (i == num - 1) ? tile_ptr[R] + nb : tile_ptr[R] + (i + 1) * len;
    }
}

// ---- encoder (main-cg-mixed.cu:2341-2346) and per-tile scaled int8 / caps ----
__device__ __forceinline__ int8_t host_trunc_i8(double v)
{
    // (int8_t)double as emitted by the x86-64 host compiler: truncate to int32
    // (0x80000000 when NaN / out of range), keep the low byte.
    int w;
    if (!(v == v) || v >= 2147483648.0 || v < -2147483648.0) w = (int)0x80000000u;
    else w = (int)v;
    return (int8_t)(unsigned char)(w & 0xFF);
}

__global__ void k_encode_ref(const double *__restrict__ tval, const float *__restrict__ tval_low, long long nnz,
                             uint16_t *__restrict__ f16, int8_t *__restrict__ i8ref)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnz; k += (long long)gridDim.x * blockDim.x) {
        f16[k] = __half_as_ushort(__float2half_rn(tval_low[k]));
        i8ref[k] = host_trunc_i8(tval[k]);
    }
}

__global__ void k_encode_tiles(const int *__restrict__ csr_offset, int tilenum, const double *__restrict__ tval,
                               int8_t *__restrict__ q, float *__restrict__ scale, unsigned char *__restrict__ caps)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < tilenum; t += gridDim.x * blockDim.x) {
        const int o = csr_offset[t], e = csr_offset[t + 1];
        double mx = 0.0, mn = INFINITY;
        bool ex32 = true, ex16 = true;
        for (int k = o; k < e; k++) {
            double a = tval[k], aa = fabs(a);
            mx = fmax(mx, aa);
            if (aa > 0.0) mn = fmin(mn, aa);
            float f = (float)a;
            if ((double)f != a) ex32 = false;
            if ((double)__half2float(__float2half_rn(f)) != a) ex16 = false;
        }
        float s = (float)(mx / 127.0);
        bool ex8 = true;
        for (int k = o; k < e; k++) {
            double a = tval[k];
            int8_t v = 0;
            if (s != 0.0f) {
                double r = rint(a / (double)s);
                r = fmin(127.0, fmax(-127.0, r));
                v = (int8_t)r;
            }
            q[k] = v;
            if ((double)((float)v * s) != a) ex8 = false;
        }
        scale[t] = s;
        unsigned char c = 0;
        if (mx <= 65504.0 && (mn == INFINITY || mn >= 6.103515625e-05)) c |= MF_CAP_FP16_OK;
        if (ex8) c |= MF_CAP_EXACT_I8;
        if (ex16) c |= MF_CAP_EXACT_F16;
        if (ex32) c |= MF_CAP_EXACT_F32;
        caps[t] = c;
    }
}

// ---- solver slices ----
__global__ void k_seg_count(const int *__restrict__ tile_ptr, int tilem, int *__restrict__ nseg)
{
    int R = blockIdx.x * blockDim.x + threadIdx.x;
    if (R >= tilem) return;
    int nt = tile_ptr[R + 1] - tile_ptr[R];
    nseg[R] = (nt + MF_SEG_TILES - 1) / MF_SEG_TILES;
}

// lane-per-row statistics of every segment: row lengths and padded width
__global__ void k_seg_shape(const int *__restrict__ tile_ptr, const int *__restrict__ seg_ptr,
                            const int *__restrict__ csr_offset, const int *__restrict__ csrptr_offset,
                            const unsigned char *__restrict__ tptr, int tilem, int rowA,
                            int *__restrict__ seg_tile0, int *__restrict__ seg_kp,
                            uint16_t *__restrict__ seg_rowlen, int *__restrict__ seg_entries,
                            long long *__restrict__ row_cost)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int i = lane & 15;
    for (int R = warp; R < tilem; R += nwarps) {
        const int rowlen = (R == tilem - 1) ? rowA - R * MF_BS : MF_BS;
        const int t0 = tile_ptr[R], t1 = tile_ptr[R + 1];
        long long cost = 4;
        for (int s = seg_ptr[R]; s < seg_ptr[R + 1]; s++) {
            const int ta = t0 + (s - seg_ptr[R]) * MF_SEG_TILES;
            const int tb = min(t1, ta + MF_SEG_TILES);
            int len = 0;
            if (i < rowlen) {
                for (int t = ta; t < tb; t++) {
                    int cc = csrptr_offset[t], nnzt = csr_offset[t + 1] - csr_offset[t];
                    int st = tptr[cc + i];
                    int sp = (i == rowlen - 1) ? nnzt : (int)tptr[cc + i + 1];
                    len += sp - st;
                }
            }
            int K = len;
            for (int o = 8; o; o >>= 1) K = max(K, __shfl_xor_sync(0xffffffffu, K, o));
            int kp = ((K + 7) / 8) * 8;
            if (kp == 0) kp = 8;
            if (lane < 16) seg_rowlen[(long long)s * MF_BS + i] = (uint16_t)len;
            if (lane == 0) {
                seg_tile0[s] = ta;
                seg_kp[s] = kp;
                seg_entries[s] = kp * MF_BS;
            }
            cost += kp + 6;
        }
        if (lane == 0) row_cost[R] = cost;
    }
}

__global__ void k_seg_fill(const int *__restrict__ tile_ptr, const int *__restrict__ seg_ptr,
                           const int *__restrict__ seg_kp, const long long *__restrict__ seg_off,
                           const int *__restrict__ csr_offset, const int *__restrict__ csrptr_offset,
                           const unsigned char *__restrict__ tptr, const unsigned char *__restrict__ tcol,
                           const double *__restrict__ tval, const float *__restrict__ tval_low,
                           const int8_t *__restrict__ q8, const int8_t *__restrict__ q8ref, int tilem, int rowA,
                           unsigned char *__restrict__ meta, double *__restrict__ v64, float *__restrict__ v32,
                           __half *__restrict__ v16, int8_t *__restrict__ v8, int8_t *__restrict__ v8ref)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int i = lane & 15;
    const int half = lane >> 4;
    for (int R = warp; R < tilem; R += nwarps) {
        const int rowlen = (R == tilem - 1) ? rowA - R * MF_BS : MF_BS;
        const int t0 = tile_ptr[R], t1 = tile_ptr[R + 1];
        const int s0 = seg_ptr[R], s1 = seg_ptr[R + 1];
        // the two half-warps take alternate segments
        for (int s = s0 + half; s < s1; s += 2) {
            const int ta = t0 + (s - s0) * MF_SEG_TILES;
            const int tb = min(t1, ta + MF_SEG_TILES);
            const int kp = seg_kp[s];
            const long long off = seg_off[s];
            int k = 0;
            if (i < rowlen) {
                for (int t = ta; t < tb; t++) {
                    int cc = csrptr_offset[t], o = csr_offset[t], nnzt = csr_offset[t + 1] - o;
                    int st = tptr[cc + i];
                    int sp = (i == rowlen - 1) ? nnzt : (int)tptr[cc + i + 1];
                    for (int e = o + st; e < o + sp; e++) {
                        meta[mf_slot<1>(off, k, i)] = (unsigned char)(((t - ta) << 4) | tcol[e]);
                        v64[mf_slot<8>(off, k, i)] = tval[e];
                        v32[mf_slot<4>(off, k, i)] = tval_low[e];
                        v16[mf_slot<2>(off, k, i)] = __float2half_rn(tval_low[e]);
                        v8[mf_slot<1>(off, k, i)] = q8[e];
                        v8ref[mf_slot<1>(off, k, i)] = q8ref[e];
                        k++;
                    }
                }
            }
            for (; k < kp; k++) {
                meta[mf_slot<1>(off, k, i)] = 0;
                v64[mf_slot<8>(off, k, i)] = 0.0;
                v32[mf_slot<4>(off, k, i)] = 0.0f;
                v16[mf_slot<2>(off, k, i)] = __float2half_rn(0.0f);
                v8[mf_slot<1>(off, k, i)] = 0;
                v8ref[mf_slot<1>(off, k, i)] = 0;
            }
        }
    }
}

// Packed per-segment header read once per segment by the solver's pipeline:
// {first tile, tile-row, Kp | ntiles << 16 | last-slice-of-tile-row << 24,
// entry offset / 128} (offsets are multiples of 128: Kp is a multiple of 8, 16 rows).
// Also writes the slice's tile words at a fixed stride of 16 per slice
// (column-tile << 8 | capability bits, 0 past the slice's tiles), so the solver
// can fetch them by slice number without waiting for the header.
__global__ void k_seg_hdr(const int *__restrict__ seg_ptr, const int *__restrict__ seg_tile0,
                          const int *__restrict__ seg_kp, const long long *__restrict__ seg_off,
                          const int *__restrict__ tile_columnidx, const unsigned char *__restrict__ caps, int tilem,
                          int4 *__restrict__ hdr, int *__restrict__ seg_tile)
{
    int R = blockIdx.x * blockDim.x + threadIdx.x;
    if (R >= tilem) return;
    for (int s = seg_ptr[R]; s < seg_ptr[R + 1]; s++) {
        const int t0 = seg_tile0[s];
        const int nt = seg_tile0[s + 1] - t0;
        const int last = (s + 1 == seg_ptr[R + 1]) ? 1 : 0;     // last slice of its tile-row
        hdr[s] = make_int4(t0, R, seg_kp[s] | (nt << 16) | (last << 24), (int)(seg_off[s] >> 7));
        for (int i = 0; i < MF_BS; i++)
            seg_tile[(long long)s * MF_BS + i] = (i < nt) ? ((tile_columnidx[t0 + i] << 8) | caps[t0 + i]) : 0;
    }
}

int grid_for(long long work, int threads)
{
    long long b = (work + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 32) b = 148 * 32;
    return (int)b;
}

template <typename T>
int dalloc(T **p, long long count, cudaStream_t s)
{
    (void)s;
    size_t bytes = (size_t)std::max<long long>(count, 1) * sizeof(T);
    MF_CUDA_TRY(cudaMalloc((void **)p, bytes));
    return MF_SUCCESS;
}

}  // namespace

#define MF_TRY(expr)                        \
    do {                                    \
        int _rc = (expr);                   \
        if (_rc != MF_SUCCESS) return _rc;  \
    } while (0)

int mf_build_tiles(mf_matrix_s *A, cudaStream_t s)
{
    auto t_start = std::chrono::steady_clock::now();
    const int rowA = A->n_rows, colA = A->n_cols;
    const int tilem = (rowA + MF_BS - 1) / MF_BS;
    const int tilen = (colA + MF_BS - 1) / MF_BS;
    A->tilem = tilem;
    A->tilen = tilen;
    A->vec_len = std::max(tilem, tilen) * MF_BS;
    int *d_err = nullptr, *d_maxes = nullptr, *d_span_base = nullptr, *d_ntiles = nullptr;
    MF_TRY(dalloc(&d_err, 1, s));
    MF_TRY(dalloc(&d_maxes, 2, s));
    MF_TRY(dalloc(&d_span_base, tilem, s));
    MF_TRY(dalloc(&d_ntiles, tilem + 1, s));
    MF_CUDA_TRY(cudaMemsetAsync(d_err, 0, sizeof(int), s));
    MF_CUDA_TRY(cudaMemsetAsync(d_maxes, 0, 2 * sizeof(int), s));
    MF_CUDA_TRY(cudaMemsetAsync(d_ntiles, 0, (tilem + 1) * sizeof(int), s));
    const int wgrid = grid_for((long long)tilem * 32, kThreads);
    if (tilem > 0) {
        k_span<<<wgrid, kThreads, 0, s>>>(A->d_rowptr, A->d_colidx, tilem, rowA, colA, d_span_base, d_maxes, d_err);
        MF_CUDA_TRY(cudaGetLastError());
    }
    int h_maxes[2] = {0, 0}, h_err = 0;
    MF_CUDA_TRY(cudaMemcpyAsync(h_maxes, d_maxes, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    if (h_err) return h_err;
    const int span = std::max(h_maxes[0], 1);
    // scratch per warp: bitmap + prefix (span words each) + tile counters (<= 32 * span)
    long long words_per_warp = 2LL * span + 32LL * span;
    int global_mode = 0;
    size_t smem = 0;
    unsigned int *gscratch = nullptr;
    int tgrid = wgrid;
    const size_t smem_cap = 96 * 1024;
    if ((size_t)words_per_warp * 4 * kWarps <= smem_cap) {
        smem = (size_t)words_per_warp * 4 * kWarps;
    } else {
        global_mode = 1;
        tgrid = 148 * 4;
        MF_TRY(dalloc(&gscratch, words_per_warp * (long long)tgrid * kWarps, s));
    }
    if (smem > 48 * 1024) {
        MF_CUDA_TRY(cudaFuncSetAttribute(k_count_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        MF_CUDA_TRY(cudaFuncSetAttribute(k_fill_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    if (tilem > 0) {
        k_count_tiles<<<tgrid, kThreads, smem, s>>>(A->d_rowptr, A->d_colidx, tilem, rowA, d_span_base, span,
                                                    (int)words_per_warp, global_mode, gscratch, d_ntiles);
        MF_CUDA_TRY(cudaGetLastError());
    }
    MF_TRY(dalloc(&A->d_tile_ptr, tilem + 1, s));
    MF_TRY(mf_scan_i32_to_i32(d_ntiles, A->d_tile_ptr, tilem, s));
    int tilenum = 0;
    MF_CUDA_TRY(cudaMemcpyAsync(&tilenum, A->d_tile_ptr + tilem, sizeof(int), cudaMemcpyDeviceToHost, s));
    int nz_lo = 0, nz_hi = 0;
    MF_CUDA_TRY(cudaMemcpyAsync(&nz_lo, A->d_rowptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaMemcpyAsync(&nz_hi, A->d_rowptr + rowA, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    const long long nnz = (long long)nz_hi - nz_lo;
    A->tilenum = tilenum;
    A->csrsize = (int)nnz;
    A->nnz = nnz;
    MF_TRY(dalloc(&A->d_tile_columnidx, tilenum + 1, s));
    MF_TRY(dalloc(&A->d_csr_offset, tilenum + 1, s));
    MF_TRY(dalloc(&A->d_csrptr_offset, tilenum + 1, s));
    MF_TRY(dalloc(&A->d_tval, nnz, s));
    MF_TRY(dalloc(&A->d_tval_low, nnz, s));
    MF_TRY(dalloc(&A->d_tcol, nnz, s));
    MF_CUDA_TRY(cudaMemsetAsync(A->d_csr_offset, 0, (tilenum + 1) * sizeof(int), s));
    MF_CUDA_TRY(cudaMemsetAsync(A->d_csrptr_offset, 0, (tilenum + 1) * sizeof(int), s));
    const long long csrptrlen_max = (long long)tilenum * MF_BS;
    MF_TRY(dalloc(&A->d_tptr, csrptrlen_max, s));
    MF_CUDA_TRY(cudaMemsetAsync(A->d_tptr, 0, (size_t)std::max<long long>(csrptrlen_max, 1), s));
    if (tilem > 0) {
        k_fill_tiles<<<tgrid, kThreads, smem, s>>>(A->d_rowptr, A->d_colidx, A->d_val, A->d_val_low, tilem, rowA,
                                                   d_span_base, span, (int)words_per_warp, global_mode, gscratch,
                                                   A->d_tile_ptr, A->d_tile_columnidx, A->d_csr_offset,
                                                   A->d_csrptr_offset, A->d_tval, A->d_tval_low, A->d_tcol,
                                                   A->d_tptr, d_err);
        MF_CUDA_TRY(cudaGetLastError());
    }
    int csrptrlen = 0;
    MF_CUDA_TRY(cudaMemcpyAsync(&csrptrlen, A->d_csrptr_offset + tilenum, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaMemcpyAsync(&h_err, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    if (h_err) return h_err;
    A->csrptrlen = csrptrlen;

    // nonempty-row lists
    int *d_nzr = nullptr;
    MF_TRY(dalloc(&d_nzr, tilenum + 1, s));
    MF_TRY(dalloc(&A->d_nonzero_row_new, tilenum + 1, s));
    MF_TRY(dalloc(&A->d_tile_rowidx, tilenum + 1, s));
    MF_TRY(dalloc(&A->d_block_signal, tilem + 4, s));
    MF_CUDA_TRY(cudaMemsetAsync(A->d_block_signal, 0, (tilem + 4) * sizeof(int), s));
    MF_CUDA_TRY(cudaMemsetAsync(d_nzr, 0, (tilenum + 1) * sizeof(int), s));
    if (tilem > 0) {
        k_rowlist_count<<<wgrid, kThreads, 0, s>>>(A->d_tile_ptr, A->d_csr_offset, A->d_csrptr_offset, A->d_tptr,
                                                   tilem, rowA, d_nzr, A->d_tile_rowidx, A->d_block_signal);
        MF_CUDA_TRY(cudaGetLastError());
    }
    MF_TRY(mf_scan_i32_to_i32(d_nzr, A->d_nonzero_row_new, tilenum, s));
    int cnt = 0;
    MF_CUDA_TRY(cudaMemcpyAsync(&cnt, A->d_nonzero_row_new + tilenum, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    A->cnt_non_new = cnt;
    MF_TRY(dalloc(&A->d_blockrowid_new, cnt + 1, s));
    MF_TRY(dalloc(&A->d_blockcsr_ptr_new, cnt + 1, s));
    MF_CUDA_TRY(cudaMemsetAsync(A->d_blockrowid_new, 0, cnt + 1, s));
    MF_CUDA_TRY(cudaMemsetAsync(A->d_blockcsr_ptr_new, 0, cnt + 1, s));
    if (tilem > 0) {
        k_rowlist_fill<<<wgrid, kThreads, 0, s>>>(A->d_tile_ptr, A->d_csr_offset, A->d_csrptr_offset, A->d_tptr,
                                                  tilem, rowA, A->d_nonzero_row_new, A->d_blockrowid_new,
                                                  A->d_blockcsr_ptr_new);
        MF_CUDA_TRY(cudaGetLastError());
    }
    // row-block split
    int *d_rbc = nullptr, *d_rbo = nullptr;
    MF_TRY(dalloc(&d_rbc, tilem + 1, s));
    MF_TRY(dalloc(&d_rbo, tilem + 1, s));
    if (tilem > 0) {
        k_rowblk_count<<<(tilem + 255) / 256, 256, 0, s>>>(A->d_tile_ptr, tilem, d_rbc);
        MF_CUDA_TRY(cudaGetLastError());
    }
    MF_TRY(mf_scan_i32_to_i32(d_rbc, d_rbo, tilem, s));
    int rb = 0;
    MF_CUDA_TRY(cudaMemcpyAsync(&rb, d_rbo + tilem, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    A->rowblkblock = rb;
    MF_TRY(dalloc(&A->d_rb_idx, rb + 1, s));
    MF_TRY(dalloc(&A->d_rb_start, rb + 1, s));
    MF_TRY(dalloc(&A->d_rb_stop, rb + 1, s));
    if (tilem > 0) {
        k_rowblk_fill<<<(tilem + 255) / 256, 256, 0, s>>>(A->d_tile_ptr, tilem, d_rbo, A->d_rb_idx, A->d_rb_start,
                                                         A->d_rb_stop);
        MF_CUDA_TRY(cudaGetLastError());
    }
    // encoder
    MF_TRY(dalloc(&A->d_val_f16, nnz, s));
    MF_TRY(dalloc(&A->d_val_i8_ref, nnz, s));
    MF_TRY(dalloc(&A->d_val_i8, nnz, s));
    MF_TRY(dalloc(&A->d_i8_scale, tilenum + 1, s));
    MF_TRY(dalloc(&A->d_tile_caps, tilenum + 1, s));
    if (nnz > 0) {
        k_encode_ref<<<grid_for(nnz, 256), 256, 0, s>>>(A->d_tval, A->d_tval_low, nnz, A->d_val_f16, A->d_val_i8_ref);
        MF_CUDA_TRY(cudaGetLastError());
    }
    if (tilenum > 0) {
        k_encode_tiles<<<grid_for(tilenum, 128), 128, 0, s>>>(A->d_csr_offset, tilenum, A->d_tval, A->d_val_i8,
                                                              A->d_i8_scale, A->d_tile_caps);
        MF_CUDA_TRY(cudaGetLastError());
    }
    // solver slices
    int *d_nseg = nullptr;
    MF_TRY(dalloc(&d_nseg, tilem + 1, s));
    MF_TRY(dalloc(&A->d_seg_ptr, tilem + 1, s));
    if (tilem > 0) {
        k_seg_count<<<(tilem + 255) / 256, 256, 0, s>>>(A->d_tile_ptr, tilem, d_nseg);
        MF_CUDA_TRY(cudaGetLastError());
    }
    MF_TRY(mf_scan_i32_to_i32(d_nseg, A->d_seg_ptr, tilem, s));
    int nseg = 0;
    MF_CUDA_TRY(cudaMemcpyAsync(&nseg, A->d_seg_ptr + tilem, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    A->nseg = nseg;
    int *d_seg_entries = nullptr;
    long long *d_cost = nullptr;
    MF_TRY(dalloc(&A->d_seg_tile0, nseg + 1, s));
    MF_TRY(dalloc(&A->d_seg_kp, nseg + 1, s));
    MF_TRY(dalloc(&A->d_seg_rowlen, (long long)nseg * MF_BS + 1, s));
    MF_TRY(dalloc(&d_seg_entries, nseg + 1, s));
    MF_TRY(dalloc(&A->d_seg_off, nseg + 1, s));
    MF_TRY(dalloc(&d_cost, tilem + 1, s));
    MF_TRY(dalloc(&A->d_row_cost, tilem + 1, s));
    if (tilem > 0) {
        k_seg_shape<<<wgrid, kThreads, 0, s>>>(A->d_tile_ptr, A->d_seg_ptr, A->d_csr_offset, A->d_csrptr_offset,
                                               A->d_tptr, tilem, rowA, A->d_seg_tile0, A->d_seg_kp,
                                               A->d_seg_rowlen, d_seg_entries, d_cost);
        MF_CUDA_TRY(cudaGetLastError());
    }
    MF_TRY(mf_scan_i32_to_i64(d_seg_entries, A->d_seg_off, nseg, s));
    MF_TRY(mf_scan_i64_to_i64(d_cost, A->d_row_cost, tilem, s));
    // seg_tile0[nseg] = tilenum (end sentinel)
    MF_CUDA_TRY(cudaMemcpyAsync(A->d_seg_tile0 + nseg, A->d_tile_ptr + tilem, sizeof(int), cudaMemcpyDeviceToDevice, s));
    MF_TRY(dalloc(&A->d_seg_hdr, nseg + 1, s));
    MF_CUDA_TRY(cudaMemsetAsync(A->d_seg_hdr, 0, (size_t)(nseg + 1) * sizeof(int4), s));
    MF_TRY(dalloc(&A->d_seg_tile, ((long long)nseg + 1) * MF_BS, s));
    if ((long long)A->tilen >= (1LL << 23)) return MF_ERR_UNSUPPORTED;   // column tile must fit 23 bits
    if (tilem > 0) {
        k_seg_hdr<<<(tilem + 255) / 256, 256, 0, s>>>(A->d_seg_ptr, A->d_seg_tile0, A->d_seg_kp, A->d_seg_off,
                                                      A->d_tile_columnidx, A->d_tile_caps, tilem, A->d_seg_hdr,
                                                      A->d_seg_tile);
        MF_CUDA_TRY(cudaGetLastError());
    }
    long long ent = 0;
    MF_CUDA_TRY(cudaMemcpyAsync(&ent, A->d_seg_off + nseg, sizeof(long long), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    A->slice_entries = ent;
    if ((ent >> 7) >= (1LL << 31)) return MF_ERR_UNSUPPORTED;
    MF_TRY(dalloc(&A->d_meta, ent, s));
    MF_TRY(dalloc(&A->d_v64, ent, s));
    MF_TRY(dalloc(&A->d_v32, ent, s));
    MF_TRY(dalloc(&A->d_v16, ent, s));
    MF_TRY(dalloc(&A->d_v8, ent, s));
    MF_TRY(dalloc(&A->d_v8ref, ent, s));
    if (tilem > 0 && nseg > 0) {
        k_seg_fill<<<wgrid, kThreads, 0, s>>>(A->d_tile_ptr, A->d_seg_ptr, A->d_seg_kp, A->d_seg_off,
                                              A->d_csr_offset, A->d_csrptr_offset, A->d_tptr, A->d_tcol, A->d_tval,
                                              A->d_tval_low, A->d_val_i8, A->d_val_i8_ref, tilem, rowA, A->d_meta,
                                              A->d_v64, A->d_v32, A->d_v16, A->d_v8, A->d_v8ref);
        MF_CUDA_TRY(cudaGetLastError());
    }
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    cudaFree(d_err); cudaFree(d_maxes); cudaFree(d_span_base); cudaFree(d_ntiles); cudaFree(d_nzr);
    cudaFree(d_rbc); cudaFree(d_rbo); cudaFree(d_nseg); cudaFree(d_seg_entries); cudaFree(d_cost);
    if (gscratch) cudaFree(gscratch);
    A->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    return MF_SUCCESS;
}
