// adjoint.cu -- what the backward pass of a differentiable solve needs beyond
// the solver itself:
//  * mf_value_grad: dL/dA on A's stored pattern, grad[e] = -sum_k lambda_k[i] x_k[j]
//    for every stored entry e = (i, j), in the caller's CSR entry order
//    (A x = b  =>  dL/dA = -lambda x^T with lambda = A^-T dL/dx);
//  * mf_matrix_create_transposed: a handle for A^T (the adjoint system of a
//    nonsymmetric A), built from A's own CSR copy.
// No counterpart in the reference, which has no differentiation.
#include "mf_internal.cuh"

#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

// One warp per row; lanes stride over the row's entries, the right-hand sides
// are summed in order (deterministic).  grad is indexed from the first stored
// entry of row 0 (rowptr[0]), like the handle's nnz.
__global__ void k_value_grad(const int *__restrict__ rowptr, const int *__restrict__ colidx, int n_rows, int n_cols,
                             int nrhs, const double *__restrict__ lambda, const double *__restrict__ x,
                             double *__restrict__ grad)
{
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int base = rowptr[0];
    for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n_rows; i += nw) {
        const int a = rowptr[i], b = rowptr[i + 1];
        for (int e = a + lane; e < b; e += 32) {
            const int j = colidx[e];
            double g = 0.0;
            for (int k = 0; k < nrhs; k++)
                g += lambda[(long long)k * n_rows + i] * x[(long long)k * n_cols + j];
            grad[e - base] = -g;
        }
    }
}

}  // namespace

extern "C" int mf_value_grad(mf_matrix A, int nrhs, const double *lambda, const double *x, double *grad_val,
                             int device_ptrs, void *stream)
{
    if (!A || !lambda || !x || !grad_val || nrhs < 1) return MF_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t nl = (size_t)nrhs * A->n_rows, nx = (size_t)nrhs * A->n_cols, ne = (size_t)A->nnz;
    const double *dl = lambda, *dx = x;
    double *dg = grad_val, *tmp = nullptr;
    if (!device_ptrs) {
        MF_CUDA_TRY(cudaMallocAsync((void **)&tmp, (nl + nx + ne) * sizeof(double) + 16, s));
        MF_CUDA_TRY(cudaMemcpyAsync(tmp, lambda, nl * sizeof(double), cudaMemcpyHostToDevice, s));
        MF_CUDA_TRY(cudaMemcpyAsync(tmp + nl, x, nx * sizeof(double), cudaMemcpyHostToDevice, s));
        dl = tmp;
        dx = tmp + nl;
        dg = tmp + nl + nx;
    }
    if (A->n_rows > 0 && ne > 0) {
        const int threads = 256;
        int blocks = (int)((A->n_rows + 7) / 8);
        if (blocks > 148 * 16) blocks = 148 * 16;
        k_value_grad<<<blocks, threads, 0, s>>>(A->d_rowptr, A->d_colidx, A->n_rows, A->n_cols, nrhs, dl, dx, dg);
        MF_CUDA_TRY(cudaGetLastError());
    }
    if (!device_ptrs) {
        MF_CUDA_TRY(cudaMemcpyAsync(grad_val, dg, ne * sizeof(double), cudaMemcpyDeviceToHost, s));
        MF_CUDA_TRY(cudaFreeAsync(tmp, s));
    }
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    return MF_SUCCESS;
}

// A^T from A's device CSR copy: a stable counting sort by column on the host
// (entries of a row of A^T keep the order of A's rows, so the result does not
// depend on scheduling), then the usual GPU tiling.
extern "C" int mf_matrix_create_transposed(mf_matrix *out, mf_matrix A, void *stream)
{
    if (!out || !A) return MF_ERR_INVALID;
    *out = nullptr;
    cudaStream_t s = (cudaStream_t)stream;
    const int m = A->n_rows, n = A->n_cols;
    const long long nnz = A->nnz;
    std::vector<int> rp(m + 1), ci(nnz > 0 ? nnz : 1);
    std::vector<double> va(nnz > 0 ? nnz : 1);
    std::vector<float> vl(nnz > 0 ? nnz : 1);
    MF_CUDA_TRY(cudaMemcpyAsync(rp.data(), A->d_rowptr, (m + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    const long long base = rp[0];   // entries of rows [0, m) start here
    if (nnz > 0) {
        MF_CUDA_TRY(cudaMemcpyAsync(ci.data(), A->d_colidx + base, nnz * sizeof(int), cudaMemcpyDeviceToHost, s));
        MF_CUDA_TRY(cudaMemcpyAsync(va.data(), A->d_val + base, nnz * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (A->d_val_low)
            MF_CUDA_TRY(cudaMemcpyAsync(vl.data(), A->d_val_low + base, nnz * sizeof(float), cudaMemcpyDeviceToHost, s));
    }
    MF_CUDA_TRY(cudaStreamSynchronize(s));
    if (!A->d_val_low)
        for (long long e = 0; e < nnz; e++) vl[e] = (float)va[e];
    std::vector<int> tp(n + 1, 0), tc(nnz > 0 ? nnz : 1);
    std::vector<double> tv(nnz > 0 ? nnz : 1);
    std::vector<float> tl(nnz > 0 ? nnz : 1);
    for (long long e = 0; e < nnz; e++) {
        if (ci[e] < 0 || ci[e] >= n) return MF_ERR_INVALID;
        tp[ci[e] + 1]++;
    }
    for (int j = 0; j < n; j++) tp[j + 1] += tp[j];
    std::vector<int> cur(tp.begin(), tp.end() - 1);
    for (int i = 0; i < m; i++)
        for (long long e = rp[i] - base; e < rp[i + 1] - base; e++) {
            const int d = cur[ci[e]]++;
            tc[d] = i;
            tv[d] = va[e];
            tl[d] = vl[e];
        }
    return mf_matrix_create(out, n, m, nnz, tp.data(), tc.data(), tv.data(), tl.data(), 0, stream);
}
