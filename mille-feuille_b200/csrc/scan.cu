// scan.cu -- device exclusive prefix sums used by the GPU tiler.
// out[0..n] with out[0] = 0 and out[n] = total (the form of the reference's
// exclusive_scan over length n+1, utils.h:34-49).  Three passes: per-block
// scan with block totals, recursive scan of the totals, add-back.
#include "mf_internal.cuh"

#include <vector>

namespace {

constexpr int kThreads = 512;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;

template <typename TI, typename TO>
__global__ void k_block_scan(const TI *__restrict__ in, TO *__restrict__ out, TO *__restrict__ block_sums,
                             long long n)
{
    __shared__ TO warp_tot[kThreads / 32];
    const long long base = (long long)blockIdx.x * kTile + (long long)threadIdx.x * kItems;
    TO v[kItems];
    TO run = 0;
#pragma unroll
    for (int j = 0; j < kItems; j++) {
        long long i = base + j;
        TO x = (i < n) ? (TO)in[i] : (TO)0;
        v[j] = run;
        run += x;
    }
    // exclusive scan of per-thread totals across the block
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    TO incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        TO t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        TO w = (lane < kThreads / 32) ? warp_tot[lane] : (TO)0;
        TO wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            TO t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < kThreads / 32) warp_tot[lane] = wi - w;   // exclusive warp offsets
        if (lane == kThreads / 32 - 1 && block_sums) block_sums[blockIdx.x] = wi;
    }
    __syncthreads();
    TO off = warp_tot[wid] + incl - run;
#pragma unroll
    for (int j = 0; j < kItems; j++) {
        long long i = base + j;
        if (i < n) out[i] = v[j] + off;
    }
}

template <typename TO>
__global__ void k_add_offsets(TO *out, const TO *block_off, long long n)
{
    const long long base = (long long)blockIdx.x * kTile;
    const TO o = block_off[blockIdx.x];
    for (int j = threadIdx.x; j < kTile; j += kThreads) {
        long long i = base + j;
        if (i < n) out[i] += o;
    }
}

template <typename TO>
__global__ void k_set_total(TO *out, long long n, const TO *block_sums_scanned, long long nb)
{
    // out[n] = total = scanned block offsets [nb]
    out[n] = block_sums_scanned[nb];
}

template <typename TI, typename TO>
int scan_impl(const TI *d_in, TO *d_out, long long n, cudaStream_t s)
{
    if (n <= 0) {
        MF_CUDA_TRY(cudaMemsetAsync(d_out, 0, sizeof(TO), s));
        return MF_SUCCESS;
    }
    long long nb = (n + kTile - 1) / kTile;
    TO *sums = nullptr, *sums_scanned = nullptr;
    MF_CUDA_TRY(cudaMallocAsync((void **)&sums, (size_t)(nb + 1) * sizeof(TO), s));
    MF_CUDA_TRY(cudaMallocAsync((void **)&sums_scanned, (size_t)(nb + 1) * sizeof(TO), s));
    k_block_scan<TI, TO><<<(unsigned)nb, kThreads, 0, s>>>(d_in, d_out, sums, n);
    MF_CUDA_TRY(cudaGetLastError());
    int rc;
    if (nb == 1) {
        MF_CUDA_TRY(cudaMemsetAsync(sums_scanned, 0, sizeof(TO), s));
        MF_CUDA_TRY(cudaMemcpyAsync(sums_scanned + 1, sums, sizeof(TO), cudaMemcpyDeviceToDevice, s));
        rc = MF_SUCCESS;
    } else {
        rc = scan_impl<TO, TO>(sums, sums_scanned, nb, s);
    }
    if (rc == MF_SUCCESS) {
        if (nb > 1) {
            k_add_offsets<TO><<<(unsigned)nb, kThreads, 0, s>>>(d_out, sums_scanned, n);
            MF_CUDA_TRY(cudaGetLastError());
        }
        k_set_total<TO><<<1, 1, 0, s>>>(d_out, n, sums_scanned, nb);
        MF_CUDA_TRY(cudaGetLastError());
    }
    MF_CUDA_TRY(cudaFreeAsync(sums, s));
    MF_CUDA_TRY(cudaFreeAsync(sums_scanned, s));
    return rc;
}

}  // namespace

int mf_scan_i32_to_i32(const int *d_in, int *d_out, long long n, cudaStream_t s)
{
    return scan_impl<int, int>(d_in, d_out, n, s);
}
int mf_scan_i32_to_i64(const int *d_in, long long *d_out, long long n, cudaStream_t s)
{
    return scan_impl<int, long long>(d_in, d_out, n, s);
}
int mf_scan_i64_to_i64(const long long *d_in, long long *d_out, long long n, cudaStream_t s)
{
    return scan_impl<long long, long long>(d_in, d_out, n, s);
}
