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
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    const int e = ro[i + 1];
    for (int k = ro[i]; k < e; ++k) s += va[k] * __ldg(x + co[k]);
    y[i] = s;
}
}  // namespace

void spmv_fp64(cfdxg_context* ctx, const cfdxg_matrix* A, const double* x, double* y) {
    ProfScope ps(ctx, "spmv_fp64", 12.0 * A->nnz + 4.0 * (A->n + 1) + 16.0 * A->n);
    launch_pdl(ctx->stream, k_spmv64, blocks_for(A->n, kT), kT, static_cast<int>(A->n), A->ro.get(), A->co.get(),
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

int prof_begin(cfdxg_context* ctx, const char* name, double bytes) {
    Profiler& P = ctx->prof;
    if (!P.on) return -1;
    cudaStreamCaptureStatus cs;
    if (cudaStreamIsCapturing(ctx->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return -1;
    int idx = -1;
    for (std::size_t k = 0; k < P.stats.size(); ++k)
        if (P.stats[k].name == name) { idx = static_cast<int>(k); break; }
    if (idx < 0) {
        P.stats.push_back(KernelStats{name});
        idx = static_cast<int>(P.stats.size()) - 1;
    }
    if (P.pool.size() < 2) {
        for (int k = 0; k < 64; ++k) {
            cudaEvent_t e;
            CFDXG_CUDA(cudaEventCreate(&e));
            P.pool.push_back(e);
        }
    }
    Profiler::Pending pe{idx, P.pool.back(), P.pool[P.pool.size() - 2], bytes};
    P.pool.pop_back();
    P.pool.pop_back();
    CFDXG_CUDA(cudaEventRecord(pe.a, ctx->stream));
    P.pending.push_back(pe);
    return static_cast<int>(P.pending.size()) - 1;
}

void prof_end(cfdxg_context* ctx, int token) {
    if (token < 0) return;
    Profiler& P = ctx->prof;
    cudaEventRecord(P.pending[token].b, ctx->stream);
    if (P.pending.size() > 4096) prof_flush(ctx);
}

void prof_flush(cfdxg_context* ctx) {
    Profiler& P = ctx->prof;
    if (P.pending.empty()) return;
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    for (const auto& pe : P.pending) {
        float ms = 0.0f;
        CFDXG_CUDA(cudaEventElapsedTime(&ms, pe.a, pe.b));
        auto& st = P.stats[pe.idx];
        ++st.launches;
        st.ms += ms;
        st.bytes += pe.bytes;
        P.pool.push_back(pe.a);
        P.pool.push_back(pe.b);
    }
    P.pending.clear();
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
