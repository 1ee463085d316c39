// solver.cu -- the persistent single-kernel CG / BiCGSTAB and the tile SpMV.
//
// One cooperative launch runs the whole solve (the reference's single-kernel
// design, Mille-feuille-cg.h:1113-1348 / main-cg-mixed.cu:1016-1385 /
// main-bicg-mixed.cu:122-723), re-designed for sm_100a:
//  * grid = SMs x resident blocks (cooperative launch guarantees co-residency);
//  * a half-warp owns a contiguous range of tile-rows (lane i = row 16R+i) for
//    every phase, so y rows are written by their owner only (no y atomics) and
//    every dot product is reduced in a fixed order (deterministic);
//  * the grid barrier is a monotone counter: red.release.gpu arrive, polled with
//    ld.acquire.gpu, every wait bounded by %globaltimer (MF_ERR_TIMEOUT);
//  * dot products: warp shuffle tree -> per-block partial in a fixed slot ->
//    after the barrier each block sums the partials in the same order;
//  * matrix payload is streamed with evict-first loads; vectors stay L2-friendly.
#include "mf_internal.cuh"

#include <cmath>
#include <cstring>
#include <vector>

namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;
constexpr int kRedKinds = 8;      // reduction slot groups
constexpr int kRedWidth = 4;      // doubles per group per block

enum { MODE_FP64 = 0, MODE_MIXED = 1, MODE_PARITY = 2 };

struct SolverParams {
    int n, tilem, vec_len;
    const int *seg_ptr, *seg_tile0, *seg_kp;
    const long long *seg_off;
    const uint16_t *seg_rowlen;
    const unsigned char *meta;
    const double *v64;
    const float *v32;
    const __half *v16;
    const int8_t *v8;
    const int *tile_col;
    const int *tile_off;          // csr_offset: tile payload offsets (tile nnz for the counters)
    const float *i8_scale;
    const unsigned char *tile_caps;
    const int *hw_begin;
    const double *b;
    double *x, *r, *p, *q, *rh, *s, *t;
    float *p32, *s32, *mag_p, *mag_s;
    signed char *lab_p, *lab_s;
    double *red;
    unsigned int *bar;
    int *err;
    double *out;
    unsigned long long *counts;
    int method, max_iter, fixed_iters, replace_every, use_lossless;
    double tol;
    float demote16, demote8;
    unsigned long long timeout_ns;
    int stall_first_barrier;   // test hook: first barrier expects one extra arrival
};

struct Shared {
    int xb[kWarps * 32];
    float sc[kWarps * 32];
    signed char pr[kWarps * 32];
    double wred[kWarps][kRedWidth];
    double bcast[kRedWidth];
    int flag;
};

// ------------------------------------------------------------ grid barrier
__device__ bool grid_barrier(const SolverParams &P, unsigned &epoch, Shared &sh)
{
    __syncthreads();
    epoch += 1;
    if (threadIdx.x == 0) {
        const unsigned target = epoch * gridDim.x + ((P.stall_first_barrier && epoch == 1) ? 1u : 0u);
        __threadfence();
        mf_red_release_add_u32(P.bar, 1u);
        bool ok = true;
        const unsigned long long t0 = mf_globaltimer();
        unsigned spins = 0;
        for (;;) {
            unsigned v = mf_ld_acquire_u32(P.bar);
            if ((int)(v - target) >= 0) break;
            if (*(volatile int *)P.err) { ok = false; break; }
            if ((++spins & 63u) == 0u && mf_globaltimer() - t0 > P.timeout_ns) {
                atomicCAS(P.err, 0, MF_ERR_TIMEOUT);
                ok = false;
                break;
            }
        }
        __threadfence();
        sh.flag = ok ? 1 : 0;
    }
    __syncthreads();
    return sh.flag != 0;
}

// Block partial of up to 4 sums (mask bit k set -> max instead of sum) written
// to red[kind][block][k].
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
            double a = (lane < kWarps) ? sh.wred[lane][k] : 0.0;
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                double b = __shfl_xor_sync(0xffffffffu, a, o);
                a = mx ? fmax(a, b) : a + b;
            }
            if (lane == 0) P.red[((long long)kind * gridDim.x + blockIdx.x) * kRedWidth + k] = a;
        }
    }
}

// After the barrier: every block sums the partials of `kind` in the same order.
__device__ void grid_collect(const SolverParams &P, Shared &sh, int kind, int nv, unsigned maxmask,
                             double *outv)
{
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    if (wib == 0) {
        for (int k = 0; k < nv; k++) {
            const bool mx = (maxmask >> k) & 1u;
            double a = 0.0;
            for (int c = lane; c < (int)gridDim.x; c += 32) {
                double b = P.red[((long long)kind * gridDim.x + c) * kRedWidth + k];
                a = mx ? fmax(a, b) : a + b;
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                double b = __shfl_xor_sync(0xffffffffu, a, o);
                a = mx ? fmax(a, b) : a + b;
            }
            if (lane == 0) sh.bcast[k] = a;
        }
    }
    __syncthreads();
    for (int k = 0; k < nv; k++) outv[k] = sh.bcast[k];
    __syncthreads();
}

// ------------------------------------------------------------ tile SpMV row
// Reference-rule label code (d_vis) -> entry precision.
__device__ __forceinline__ int parity_prec(int code)
{
    return code == 0 ? MF_P64 : code == 4 ? MF_P32 : code == 3 ? MF_P16 : code == 2 ? MF_P8 : MF_PSKIP;
}

// y for row 16R+i of the half-warp's tile-row R.  force_pr >= 0 forces one
// precision for every tile (used by the FP64 residual replacement and SpMV).
template <int MODE>
__device__ __forceinline__ double spmv_row(const SolverParams &P, Shared &sh, int R, int i, int tb, unsigned hmask,
                                           const double *x64, const float *x32, const float *mag, float invM,
                                           const signed char *lab, int force_pr, unsigned long long *cnt)
{
    double acc = 0.0;
    const int s_beg = P.seg_ptr[R], s_end = P.seg_ptr[R + 1];
    for (int s = s_beg; s < s_end; s++) {
        const int t0 = P.seg_tile0[s];
        const int nt = P.seg_tile0[s + 1] - t0 < MF_SEG_TILES ? P.seg_tile0[s + 1] - t0 : MF_SEG_TILES;
        if (i < nt) {
            const int t = t0 + i;
            const int jc = P.tile_col[t];
            int pr;
            if (force_pr >= 0 || MODE == MODE_FP64) {
                pr = force_pr >= 0 ? force_pr : MF_P64;
            } else if (MODE == MODE_MIXED) {
                const unsigned cap = P.tile_caps[t];
                const float rel = mag[jc] * invM;
                pr = MF_P32;
                if (rel <= P.demote8) pr = MF_P8;
                else if (rel <= P.demote16 && (cap & MF_CAP_FP16_OK)) pr = MF_P16;
                if (P.use_lossless) {
                    if (cap & MF_CAP_EXACT_I8) pr = MF_P8;
                    else if ((cap & MF_CAP_EXACT_F16) && pr == MF_P32) pr = MF_P16;
                }
            } else {
                pr = parity_prec(lab[jc]);
            }
            sh.xb[tb + i] = jc * MF_BS;
            sh.pr[tb + i] = (signed char)pr;
            sh.sc[tb + i] = P.i8_scale[t];
            if (cnt) {
                const unsigned long long nz = (unsigned long long)(P.tile_off[t + 1] - P.tile_off[t]);
#pragma unroll
                for (int j = 0; j < 5; j++) {
                    cnt[j] += (pr == j) ? 1ull : 0ull;       // tile products per precision
                    cnt[5 + j] += (pr == j) ? nz : 0ull;     // entries per precision
                }
            }
        }
        __syncwarp(hmask);
        const long long off = P.seg_off[s];
        const int kp = P.seg_kp[s];
        const int len = P.seg_rowlen[(long long)s * MF_BS + i];
        const unsigned long long *mrow = (const unsigned long long *)(P.meta + off + (long long)i * kp);
        float part = 0.0f;
        int prev = -1;
        for (int k0 = 0; k0 < len; k0 += 8) {
            const unsigned long long m8 = __ldcs(mrow + (k0 >> 3));
            if (MODE == MODE_FP64 || force_pr == MF_P64) {
                double vv[8], xx[8];
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const int k = k0 + j;
                    const unsigned mm = (unsigned)(m8 >> (8 * j)) & 0xFFu;
                    const long long e = off + (long long)k * MF_BS + i;
                    if (k < len) {
                        vv[j] = __ldcs(P.v64 + e);
                        xx[j] = x64[sh.xb[tb + (mm >> 4)] + (mm & 15u)];
                    } else {
                        vv[j] = 0.0;
                        xx[j] = 0.0;
                    }
                }
#pragma unroll
                for (int j = 0; j < 8; j++) acc = fma(vv[j], xx[j], acc);
            } else {
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const int k = k0 + j;
                    if (k >= len) break;
                    const unsigned mm = (unsigned)(m8 >> (8 * j)) & 0xFFu;
                    const int slot = (int)(mm >> 4);
                    const long long e = off + (long long)k * MF_BS + i;
                    const int xi = sh.xb[tb + slot] + (int)(mm & 15u);
                    const int pr = sh.pr[tb + slot];
                    if (slot != prev) {
                        acc += (double)part;
                        part = 0.0f;
                        prev = slot;
                    }
                    if (pr == MF_P64) {
                        acc = fma(__ldcs(P.v64 + e), x64[xi], acc);
                    } else if (pr == MF_P32) {
                        part = fmaf(__ldcs(P.v32 + e), x32[xi], part);
                    } else if (pr == MF_P16) {
                        part = fmaf(__half2float(P.v16[e]), x32[xi], part);
                    } else if (pr == MF_P8) {
                        part = fmaf((float)P.v8[e] * sh.sc[tb + slot], x32[xi], part);
                    }
                }
            }
        }
        acc += (double)part;
        __syncwarp(hmask);
    }
    return acc;
}

// ------------------------------------------------------------ phases
struct Ctx {
    int lane, wib, half, i, tb, rbeg, rend;
    unsigned hmask;
};

__device__ __forceinline__ Ctx make_ctx(const SolverParams &P)
{
    Ctx c;
    c.lane = threadIdx.x & 31;
    c.wib = threadIdx.x >> 5;
    c.half = c.lane >> 4;
    c.i = c.lane & 15;
    c.tb = c.wib * 32 + c.half * 16;
    c.hmask = 0xFFFFu << (16 * c.half);
    const int hw = (blockIdx.x * kWarps + c.wib) * 2 + c.half;
    c.rbeg = P.hw_begin[hw];
    c.rend = P.hw_begin[hw + 1];
    return c;
}

// max over the 16 lanes of a half-warp
// max over the 16 lanes of a half-warp; hmask names exactly those lanes (the
// two halves of a warp walk different tile-row ranges, so they never shuffle together)
__device__ __forceinline__ float half_max(float v, unsigned hmask)
{
#pragma unroll
    for (int o = 8; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(hmask, v, o));
    return v;
}
__device__ __forceinline__ int half_max_i(int v, unsigned hmask)
{
#pragma unroll
    for (int o = 8; o; o >>= 1) v = max(v, __shfl_xor_sync(hmask, v, o));
    return v;
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

// Write a direction vector's FP32 shadow and segment statistics for the rows
// of tile-row R (all 16 lanes of the half-warp call this together).
template <int MODE>
__device__ __forceinline__ void publish_dir(const SolverParams &P, int R, int row, bool valid, double vnew,
                                            double vold, float *v32, float *mag, signed char *lab, float &bmax,
                                            unsigned hmask, bool labels)
{
    if (valid) v32[row] = (float)vnew;
    if (MODE == MODE_MIXED) {
        float m = half_max(valid ? (float)fabs(vnew) : 0.0f, hmask);
        bmax = fmaxf(bmax, m);
        if ((threadIdx.x & 15) == 0) mag[R] = m;
    } else if (MODE == MODE_PARITY && labels) {
        // reference rule: label of the next SpMV's tile column from |v_new - v_old|
        int rk = half_max_i(valid ? ref_rank(fabs(vnew - vold)) : 0, hmask);
        if ((threadIdx.x & 15) == 0) lab[R] = rank_to_vis(rk);
    }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, 2) k_solve(SolverParams P)
{
    __shared__ Shared sh;
    const Ctx c = make_ctx(P);
    unsigned epoch = 0;
    unsigned long long cnt[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int n = P.n;
    const bool bicg = (P.method == MF_METHOD_BICGSTAB);

    // ---- init: x = 0 (owned rows), r = b, p = r (rh = r) ----
    double pb = 0.0, pr1 = 0.0;
    float bmax = 0.0f;
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
        publish_dir<MODE>(P, R, row, valid, bv, 0.0, P.p32, P.mag_p, P.lab_p, bmax, c.hmask, false);
        pb += bv * bv;
    }
    pr1 = pb;
    block_partial(P, sh, 0, pb, pr1, (double)bmax, 0.0, 3, 0x4u);
    if (!grid_barrier(P, epoch, sh)) return;
    double v[4];
    grid_collect(P, sh, 0, 3, 0x4u, v);
    const double bb = v[0];
    double rr = v[0], r1 = v[1];
    float invM = v[2] > 0.0 ? (float)(1.0 / v[2]) : 0.0f;
    float invMs = 0.0f;
    // parity mode: initial labels are all FP64 (cudaMemset(d_vis, 0), main-cg-mixed.cu:2828)
    const double thr2 = P.tol * P.tol * bb;
    int k = 0, conv = 0, repl = 0, status = 0, last_true = 0;
    double rr_true = rr;
    if (!P.fixed_iters && rr <= thr2) { conv = 1; last_true = 1; }

    // reference labels start at FP64 for p (d_vis zeroed)
    while (!conv && k < P.max_iter) {
        if (!bicg) {
            // ---- Phase A: q = A p, p.q ----
            double ppq = 0.0;
            for (int R = c.rbeg; R < c.rend; R++) {
                const double y = spmv_row<MODE>(P, sh, R, c.i, c.tb, c.hmask, P.p, P.p32, P.mag_p, invM, P.lab_p,
                                                -1, cnt);
                const int row = R * MF_BS + c.i;
                if (row < n) {
                    P.q[row] = y;
                    ppq += P.p[row] * y;
                }
            }
            block_partial(P, sh, 1, ppq, 0, 0, 0, 1, 0u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 1, 1, 0u, v);
            const double alpha = rr / v[0];
            if (!isfinite(alpha)) { status = MF_ERR_BREAKDOWN; break; }
            // ---- Phase B: x += alpha p, r -= alpha q, r.r ----
            double prr = 0.0;
            for (int R = c.rbeg; R < c.rend; R++) {
                const int row = R * MF_BS + c.i;
                if (row < n) {
                    P.x[row] += alpha * P.p[row];
                    const double rv = P.r[row] - alpha * P.q[row];
                    P.r[row] = rv;
                    prr += rv * rv;
                }
            }
            block_partial(P, sh, 2, prr, 0, 0, 0, 1, 0u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 2, 1, 0u, v);
            double rr_new = v[0];
            k++;
            last_true = 0;
            const bool want_check = !P.fixed_iters && rr_new <= thr2;
            const bool want_repl = P.replace_every > 0 && (k % P.replace_every) == 0;
            if (want_check || want_repl) {
                // ---- FP64 true residual: r = b - A x ----
                double prt = 0.0;
                for (int R = c.rbeg; R < c.rend; R++) {
                    const double y = spmv_row<MODE>(P, sh, R, c.i, c.tb, c.hmask, P.x, nullptr, nullptr, 0.f,
                                                    nullptr, MF_P64, nullptr);
                    const int row = R * MF_BS + c.i;
                    if (row < n) {
                        const double rv = P.b[row] - y;
                        P.r[row] = rv;
                        prt += rv * rv;
                    }
                }
                block_partial(P, sh, 3, prt, 0, 0, 0, 1, 0u);
                if (!grid_barrier(P, epoch, sh)) return;
                grid_collect(P, sh, 3, 1, 0u, v);
                rr_new = v[0];
                rr_true = rr_new;
                repl++;
                last_true = 1;
                if (!P.fixed_iters && rr_new <= thr2) { rr = rr_new; conv = 1; break; }
            }
            const double beta = rr_new / rr;
            rr = rr_new;
            // ---- Phase C: p = r + beta p ----
            bmax = 0.0f;
            for (int R = c.rbeg; R < c.rend; R++) {
                const int row = R * MF_BS + c.i;
                const bool valid = row < n;
                double pold = 0.0, pn = 0.0;
                if (valid) {
                    pold = P.p[row];
                    pn = P.r[row] + beta * pold;
                    P.p[row] = pn;
                }
                publish_dir<MODE>(P, R, row, valid, pn, pold, P.p32, P.mag_p, P.lab_p, bmax, c.hmask, true);
            }
            block_partial(P, sh, 4, (double)bmax, 0, 0, 0, 1, 0x1u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 4, 1, 0x1u, v);
            invM = v[0] > 0.0 ? (float)(1.0 / v[0]) : 0.0f;
        } else {
            // ---- BiCGSTAB: v = A p, alpha = r1 / (rh.v) ----
            double prv = 0.0;
            for (int R = c.rbeg; R < c.rend; R++) {
                const double y = spmv_row<MODE>(P, sh, R, c.i, c.tb, c.hmask, P.p, P.p32, P.mag_p, invM, P.lab_p,
                                                -1, cnt);
                const int row = R * MF_BS + c.i;
                if (row < n) {
                    P.q[row] = y;
                    prv += P.rh[row] * y;
                }
            }
            block_partial(P, sh, 1, prv, 0, 0, 0, 1, 0u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 1, 1, 0u, v);
            const double alpha = r1 / v[0];
            if (!isfinite(alpha)) { status = MF_ERR_BREAKDOWN; break; }
            // s = r - alpha v
            float smax = 0.0f;
            for (int R = c.rbeg; R < c.rend; R++) {
                const int row = R * MF_BS + c.i;
                const bool valid = row < n;
                double sold = 0.0, sn = 0.0;
                if (valid) {
                    sold = P.s[row];
                    sn = P.r[row] - alpha * P.q[row];
                    P.s[row] = sn;
                }
                publish_dir<MODE>(P, R, row, valid, sn, sold, P.s32, P.mag_s, P.lab_s, smax, c.hmask, true);
            }
            block_partial(P, sh, 2, (double)smax, 0, 0, 0, 1, 0x1u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 2, 1, 0x1u, v);
            invMs = v[0] > 0.0 ? (float)(1.0 / v[0]) : 0.0f;
            // t = A s, omega = (t.s)/(t.t)
            double pts = 0.0, ptt = 0.0;
            for (int R = c.rbeg; R < c.rend; R++) {
                const double y = spmv_row<MODE>(P, sh, R, c.i, c.tb, c.hmask, P.s, P.s32, P.mag_s, invMs, P.lab_s,
                                                -1, cnt);
                const int row = R * MF_BS + c.i;
                if (row < n) {
                    P.t[row] = y;
                    pts += y * P.s[row];
                    ptt += y * y;
                }
            }
            block_partial(P, sh, 3, pts, ptt, 0, 0, 2, 0u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 3, 2, 0u, v);
            const double omega = (v[1] != 0.0) ? v[0] / v[1] : 0.0;
            // x += alpha p + omega s; r = s - omega t
            double prr = 0.0, prh = 0.0;
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
            block_partial(P, sh, 4, prr, prh, 0, 0, 2, 0u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 4, 2, 0u, v);
            double rr_new = v[0], r1_new = v[1];
            k++;
            last_true = 0;
            const bool want_check = !P.fixed_iters && rr_new <= thr2;
            const bool want_repl = P.replace_every > 0 && (k % P.replace_every) == 0;
            if (want_check || want_repl) {
                double prt = 0.0, prth = 0.0;
                for (int R = c.rbeg; R < c.rend; R++) {
                    const double y = spmv_row<MODE>(P, sh, R, c.i, c.tb, c.hmask, P.x, nullptr, nullptr, 0.f,
                                                    nullptr, MF_P64, nullptr);
                    const int row = R * MF_BS + c.i;
                    if (row < n) {
                        const double rv = P.b[row] - y;
                        P.r[row] = rv;
                        prt += rv * rv;
                        prth += rv * P.rh[row];
                    }
                }
                block_partial(P, sh, 5, prt, prth, 0, 0, 2, 0u);
                if (!grid_barrier(P, epoch, sh)) return;
                grid_collect(P, sh, 5, 2, 0u, v);
                rr_new = v[0];
                r1_new = v[1];
                rr_true = rr_new;
                repl++;
                last_true = 1;
                if (!P.fixed_iters && rr_new <= thr2) { rr = rr_new; conv = 1; break; }
            }
            const double beta = (r1_new * alpha) / (r1 * omega);
            rr = rr_new;
            r1 = r1_new;
            if (!isfinite(beta)) { status = MF_ERR_BREAKDOWN; break; }
            // p = r + beta (p - omega v)
            bmax = 0.0f;
            for (int R = c.rbeg; R < c.rend; R++) {
                const int row = R * MF_BS + c.i;
                const bool valid = row < n;
                double pold = 0.0, pn = 0.0;
                if (valid) {
                    pold = P.p[row];
                    pn = P.r[row] + beta * (pold - omega * P.q[row]);
                    P.p[row] = pn;
                }
                publish_dir<MODE>(P, R, row, valid, pn, pold, P.p32, P.mag_p, P.lab_p, bmax, c.hmask, true);
            }
            block_partial(P, sh, 6, (double)bmax, 0, 0, 0, 1, 0x1u);
            if (!grid_barrier(P, epoch, sh)) return;
            grid_collect(P, sh, 6, 1, 0x1u, v);
            invM = v[0] > 0.0 ? (float)(1.0 / v[0]) : 0.0f;
        }
    }
    // ---- final FP64 true residual when the last one was not already formed ----
    if (!last_true) {
        double prt = 0.0;
        for (int R = c.rbeg; R < c.rend; R++) {
            const double y = spmv_row<MODE>(P, sh, R, c.i, c.tb, c.hmask, P.x, nullptr, nullptr, 0.f, nullptr,
                                            MF_P64, nullptr);
            const int row = R * MF_BS + c.i;
            if (row < n) {
                const double d = P.b[row] - y;
                prt += d * d;
            }
        }
        block_partial(P, sh, 7, prt, 0, 0, 0, 1, 0u);
        if (!grid_barrier(P, epoch, sh)) return;
        grid_collect(P, sh, 7, 1, 0u, v);
        rr_true = v[0];
    }
    // tile-use counters
    for (int j = 0; j < 10; j++) {
        unsigned long long a = cnt[j];
        for (int o = 16; o; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (c.lane == 0 && a) atomicAdd(&P.counts[j], a);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.out[0] = (double)k;
        P.out[1] = (double)conv;
        P.out[2] = bb > 0 ? sqrt(rr_true / bb) : 0.0;
        P.out[3] = bb > 0 ? sqrt(rr / bb) : 0.0;
        P.out[4] = sqrt(rr);
        P.out[5] = (double)repl;
        P.out[6] = (double)status;
    }
}

// ------------------------------------------------------------ standalone SpMV
template <int MODE>
__global__ void __launch_bounds__(kThreads) k_spmv(SolverParams P, int force_pr, double *y)
{
    __shared__ Shared sh;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, half = lane >> 4, i = lane & 15;
    const int tb = wib * 32 + half * 16;
    const unsigned hmask = 0xFFFFu << (16 * half);
    const int hw = (blockIdx.x * kWarps + wib) * 2 + half;
    const int nhw = gridDim.x * kWarps * 2;
    for (int R = hw; R < P.tilem; R += nhw) {
        const double v = spmv_row<MODE>(P, sh, R, i, tb, hmask, P.x, P.p32, nullptr, 0.f, nullptr, force_pr,
                                        nullptr);
        const int row = R * MF_BS + i;
        if (row < P.n) y[row] = v;
    }
}

__global__ void k_to_f32(const double *x, float *y, long long n)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        y[k] = (float)x[k];
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

// ------------------------------------------------------------ workspace
struct Workspace {
    int G;                 // grid blocks of the persistent kernel
    int mode;
    double *r, *p, *q, *rh, *s, *t, *x;
    float *p32, *s32, *mag_p, *mag_s;
    signed char *lab_p, *lab_s;
    double *red;
    unsigned int *bar;
    int *err;
    double *out;
    unsigned long long *counts;
    int *hw_begin;
    int nhw;
    cudaEvent_t e0, e1;
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

const void *solve_kernel(int mode)
{
    if (mode == MODE_FP64) return (const void *)k_solve<MODE_FP64>;
    if (mode == MODE_MIXED) return (const void *)k_solve<MODE_MIXED>;
    return (const void *)k_solve<MODE_PARITY>;
}

int ws_get(mf_matrix_s *A, int mode, int blocks_per_sm, Workspace **out, cudaStream_t s)
{
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
        int o = 0;
        MF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, solve_kernel(m), kThreads, 0));
        occ = o < occ ? o : occ;
    }
    (void)mode;
    if (occ < 1) return MF_ERR_UNSUPPORTED;
    if (blocks_per_sm > 0 && blocks_per_sm < occ) occ = blocks_per_sm;
    int G = nsm * occ;
    // small systems: no more blocks than needed for one tile-row per half-warp
    const int need = (A->tilem + kWarps * 2 - 1) / (kWarps * 2);
    if (need < G) G = need > 0 ? need : 1;
    Workspace *w = (Workspace *)A->ws;
    if (w && w->G == G) {
        *out = w;
        return MF_SUCCESS;
    }
    if (w) mf_solver_free_ws(A);
    w = new Workspace();
    memset(w, 0, sizeof(*w));
    w->G = G;
    const long long L = A->vec_len;
    const long long S = std::max(A->tilem, A->tilen) + 1;
    MF_TRY(dal(&w->r, L)); MF_TRY(dal(&w->p, L)); MF_TRY(dal(&w->q, L)); MF_TRY(dal(&w->rh, L));
    MF_TRY(dal(&w->s, L)); MF_TRY(dal(&w->t, L)); MF_TRY(dal(&w->x, L));
    MF_TRY(dal(&w->p32, L)); MF_TRY(dal(&w->s32, L));
    MF_TRY(dal(&w->mag_p, S)); MF_TRY(dal(&w->mag_s, S));
    MF_TRY(dal(&w->lab_p, S)); MF_TRY(dal(&w->lab_s, S));
    MF_TRY(dal(&w->red, (long long)kRedKinds * G * kRedWidth));
    MF_TRY(dal(&w->bar, 1)); MF_TRY(dal(&w->err, 1)); MF_TRY(dal(&w->out, 16));
    MF_TRY(dal(&w->counts, 16));
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
    P.seg_ptr = A->d_seg_ptr;
    P.seg_tile0 = A->d_seg_tile0;
    P.seg_kp = A->d_seg_kp;
    P.seg_off = A->d_seg_off;
    P.seg_rowlen = A->d_seg_rowlen;
    P.meta = A->d_meta;
    P.v64 = A->d_v64;
    P.v32 = A->d_v32;
    P.v16 = A->d_v16;
    P.v8 = A->d_v8;
    P.tile_col = A->d_tile_columnidx;
    P.tile_off = A->d_csr_offset;
    P.i8_scale = A->d_i8_scale;
    P.tile_caps = A->d_tile_caps;
    if (w) {
        P.hw_begin = w->hw_begin;
        P.x = w->x; P.r = w->r; P.p = w->p; P.q = w->q; P.rh = w->rh; P.s = w->s; P.t = w->t;
        P.p32 = w->p32; P.s32 = w->s32; P.mag_p = w->mag_p; P.mag_s = w->mag_s;
        P.lab_p = w->lab_p; P.lab_s = w->lab_s;
        P.red = w->red; P.bar = w->bar; P.err = w->err; P.out = w->out; P.counts = w->counts;
    }
}

}  // namespace

void mf_solver_free_ws(mf_matrix_s *A)
{
    Workspace *w = (Workspace *)A->ws;
    if (!w) return;
    cudaFree(w->r); cudaFree(w->p); cudaFree(w->q); cudaFree(w->rh); cudaFree(w->s); cudaFree(w->t);
    cudaFree(w->x); cudaFree(w->p32); cudaFree(w->s32); cudaFree(w->mag_p); cudaFree(w->mag_s);
    cudaFree(w->lab_p); cudaFree(w->lab_s); cudaFree(w->red); cudaFree(w->bar); cudaFree(w->err);
    cudaFree(w->out); cudaFree(w->counts); cudaFree(w->hw_begin);
    cudaEventDestroy(w->e0); cudaEventDestroy(w->e1);
    delete w;
    A->ws = nullptr;
}

int mf_solver_run(mf_matrix_s *A, const double *d_b, double *d_x, const mf_options *opt, mf_report *rep,
                  cudaStream_t s)
{
    const int mode = opt->precision == MF_PREC_FP64 ? MODE_FP64
                     : opt->precision == MF_PREC_PARITY ? MODE_PARITY : MODE_MIXED;
    if (opt->method != MF_METHOD_CG && opt->method != MF_METHOD_BICGSTAB) return MF_ERR_INVALID;
    if (opt->x0_given) return MF_ERR_UNSUPPORTED;
    Workspace *w = nullptr;
    MF_TRY(ws_get(A, mode, opt->blocks_per_sm, &w, s));
    const long long L = A->vec_len;
    const long long S = std::max(A->tilem, A->tilen) + 1;
    // zero the padded tails and the state the kernel reads before writing
    MF_CUDA_TRY(cudaMemsetAsync(w->x, 0, L * sizeof(double), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->p, 0, L * sizeof(double), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->s, 0, L * sizeof(double), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->p32, 0, L * sizeof(float), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->s32, 0, L * sizeof(float), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->mag_p, 0, S * sizeof(float), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->mag_s, 0, S * sizeof(float), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->lab_p, 0, S, s));
    MF_CUDA_TRY(cudaMemsetAsync(w->lab_s, 0, S, s));
    MF_CUDA_TRY(cudaMemsetAsync(w->bar, 0, sizeof(unsigned int), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->err, 0, sizeof(int), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->out, 0, 16 * sizeof(double), s));
    MF_CUDA_TRY(cudaMemsetAsync(w->counts, 0, 16 * sizeof(unsigned long long), s));
    SolverParams P;
    fill_params(P, A, w);
    P.b = d_b;
    P.method = opt->method;
    P.max_iter = opt->max_iter;
    P.fixed_iters = opt->fixed_iters;
    P.replace_every = opt->replace_every;
    P.use_lossless = opt->use_lossless;
    P.tol = opt->tol;
    P.demote16 = (float)opt->demote_fp16;
    P.demote8 = (float)opt->demote_int8;
    double to = opt->wait_timeout_s > 0 ? opt->wait_timeout_s : 10.0;
    P.timeout_ns = (unsigned long long)(to * 1e9);
    P.stall_first_barrier = opt->test_stall_barrier ? 1 : 0;
    void *args[] = {&P};
    MF_CUDA_TRY(cudaEventRecord(w->e0, s));
    MF_CUDA_TRY(cudaLaunchCooperativeKernel(solve_kernel(mode), dim3(w->G), dim3(kThreads), args, 0, s));
    MF_CUDA_TRY(cudaEventRecord(w->e1, s));
    double out[16];
    unsigned long long counts[16];
    int err = 0;
    MF_CUDA_TRY(cudaMemcpyAsync(out, w->out, sizeof(out), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaMemcpyAsync(counts, w->counts, sizeof(counts), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaMemcpyAsync(&err, w->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaMemcpyAsync(d_x, w->x, (size_t)A->n_rows * sizeof(double), cudaMemcpyDeviceToDevice, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    float ms = 0.f;
    MF_CUDA_TRY(cudaEventElapsedTime(&ms, w->e0, w->e1));
    if (rep) {
        memset(rep, 0, sizeof(*rep));
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
    }
    if (err) return err;
    return (int)out[6];
}

int mf_spmv_run(mf_matrix_s *A, const double *d_x, double *d_y, int precision, cudaStream_t s, double *elapsed_ms)
{
    // x is read through a padded copy so that column tiles past n_rows read zeros
    Workspace *w = nullptr;
    MF_TRY(ws_get(A, MODE_FP64, 0, &w, s));
    const long long L = A->vec_len;
    MF_CUDA_TRY(cudaMemsetAsync(w->x, 0, L * sizeof(double), s));
    MF_CUDA_TRY(cudaMemcpyAsync(w->x, d_x, (size_t)A->n_cols * sizeof(double), cudaMemcpyDeviceToDevice, s));
    k_to_f32<<<256, 256, 0, s>>>(w->x, w->p32, L);
    MF_CUDA_TRY(cudaGetLastError());
    SolverParams P;
    fill_params(P, A, w);
    int nsm = 0, dev = 0;
    MF_CUDA_TRY(cudaGetDevice(&dev));
    MF_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int hw_per_block = kWarps * 2;
    int blocks = (A->tilem + hw_per_block - 1) / hw_per_block;
    const int cap = nsm * 4;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    const int fpr = precision == MF_PREC_FP64 ? MF_P64 : MF_P32;
    MF_CUDA_TRY(cudaEventRecord(w->e0, s));
    if (fpr == MF_P64) k_spmv<MODE_FP64><<<blocks, kThreads, 0, s>>>(P, MF_P64, d_y);
    else k_spmv<MODE_MIXED><<<blocks, kThreads, 0, s>>>(P, MF_P32, d_y);
    MF_CUDA_TRY(cudaGetLastError());
    MF_CUDA_TRY(cudaEventRecord(w->e1, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    if (elapsed_ms) {
        float ms = 0.f;
        MF_CUDA_TRY(cudaEventElapsedTime(&ms, w->e0, w->e1));
        *elapsed_ms = ms;
    }
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
