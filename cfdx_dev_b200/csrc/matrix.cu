// matrix.cu -- device CSR matrices, FP64 SpMV and the context status word.
#include <cmath>

#include "objects.h"

namespace cfdxg {

namespace {
constexpr int kT = 256;

// y = A x, per-row sum in CSR order from 0.0 (SparseMatrix::matvec, sparse_matrix.h:180-195).
__global__ void k_spmv64(int n, const int* __restrict__ ro, const int* __restrict__ co,
                         const double* __restrict__ va, const double* __restrict__ x,
                         double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    const int e = ro[i + 1];
    for (int k = ro[i]; k < e; ++k) s += va[k] * __ldg(x + co[k]);
    y[i] = s;
}
}  // namespace

void spmv_fp64(cfdxg_context* ctx, const cfdxg_matrix* A, const double* x, double* y) {
    k_spmv64<<<blocks_for(A->n, kT), kT, 0, ctx->stream>>>(static_cast<int>(A->n), A->ro.get(), A->co.get(),
                                                           A->va.get(), x, y);
    check_launch(ctx);
}

void matrix_sync_host_values(cfdxg_context* ctx, cfdxg_matrix* A) {
    if (A->host_values_valid) return;
    A->host.va.resize(static_cast<std::size_t>(A->nnz));
    A->va.download(A->host.va.data(), ctx->stream);
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    A->host_values_valid = true;
}

void clear_status(cfdxg_context* ctx) {
    CFDXG_CUDA(cudaMemsetAsync(ctx->scratch.status, 0, sizeof(int), ctx->stream));
}

int read_status(cfdxg_context* ctx) {
    CFDXG_CUDA(cudaMemcpyAsync(ctx->scratch.host_status, ctx->scratch.status, sizeof(int),
                               cudaMemcpyDeviceToHost, ctx->stream));
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    return *ctx->scratch.host_status;
}

}  // namespace cfdxg
