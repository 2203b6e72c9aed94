// gauge.cu -- pressure gauge of a pure-Neumann system on the device.
//
// Two forms, as the reference has them:
//
//  * elimination of a reference cell (physics/steady_incompressible_solver.h
//    :8617-8654, the pure-Neumann pressure corrector; reference cell
//    controls.pressure_reference_cell, default 0): the principal
//    submatrix without row and column `ref` (later indices shift down by one)
//    and the right-hand side without entry `ref`; after the solve the full
//    correction is the reduced one with 0 at `ref`;
//  * an identity row (core/solvers/scalar_diffusion.h:177-210
//    apply_reference_cell_gauge): row and column `ref` removed, a unit
//    diagonal at (ref, ref), rhs_i -= a_i,ref * value and rhs_ref = value.
//
// The output pattern depends only on the input pattern, so it is built once
// on the host into a plan (the output CSR and, per output entry, the input
// entry it copies); each application is then two gathers on the device --
// the values and the right-hand side -- which is what changes between SIMPLE
// iterations.
#include <vector>

#include "io.h"

struct cfdxg_gauge {
    int32_t mode = CFDXG_GAUGE_ELIMINATE;
    int64_t n = 0, ref = 0, n_out = 0, nnz_in = 0, nnz_out = 0;
    double value = 0.0;
    std::vector<uint32_t> hro, hco;      // output pattern
    cfdxg::DevBuf<int> ro, co;           // output pattern on the device
    cfdxg::DevBuf<int> src;              // nnz_out: input entry, -1 = the unit diagonal
    cfdxg::DevBuf<int> colref;           // identity row: per row the (i, ref) entry or -1
};

using namespace cfdxg;

namespace {

constexpr int kT = 256;

__global__ void k_gauge_values(int64_t nnz, const int* __restrict__ src, const double* __restrict__ va,
                               double* __restrict__ out) {
    const int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    if (k >= nnz) return;
    const int s = src[k];
    out[k] = s >= 0 ? va[s] : 1.0;
}

// elimination: rhs_out[i'] = rhs[i' < ref ? i' : i' + 1]
__global__ void k_gauge_rhs_eliminate(int n_out, int ref, const double* __restrict__ b, double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n_out) out[i] = b[i < ref ? i : i + 1];
}

// identity row: rhs_i - a_i,ref * value (a_i,ref = 0 where absent), rhs_ref = value
__global__ void k_gauge_rhs_identity(int n, int ref, double value, const int* __restrict__ colref,
                                     const double* __restrict__ va, const double* __restrict__ b,
                                     double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i == ref) {
        out[i] = value;
        return;
    }
    const int k = colref[i];
    const double a = k >= 0 ? va[k] : 0.0;
    out[i] = b[i] - a * value;
}

// full correction: x[ref] = 0, the others from the reduced solution in order
__global__ void k_gauge_expand(int n, int ref, const double* __restrict__ xr, double* __restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] = i == ref ? 0.0 : xr[i < ref ? i : i - 1];
}

}  // namespace

extern "C" int cfdxg_gauge_create(cfdxg_context* ctx, const cfdxg_matrix* A, int32_t mode, int64_t ref,
                                  double value, cfdxg_gauge** out) {
    if (!ctx) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    if (!A || !out) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "missing argument");
    if (mode != CFDXG_GAUGE_ELIMINATE && mode != CFDXG_GAUGE_IDENTITY_ROW)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "unknown gauge mode");
    const int64_t n = A->n;
    if (ref < 0 || ref >= n) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "reference cell out of range");
    if (mode == CFDXG_GAUGE_ELIMINATE && n == 1)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT,
                    "eliminating the only unknown leaves an empty system (keep the trivial equation p = 0)");
    if (mode == CFDXG_GAUGE_IDENTITY_ROW && !std::isfinite(value))
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "reference value must be finite");
    auto g = std::make_unique<cfdxg_gauge>();
    g->mode = mode;
    g->n = n;
    g->ref = ref;
    g->value = value;
    g->nnz_in = A->nnz;
    const HostCsr& H = A->host;   // the pattern mirror is always valid
    std::vector<int> src, colref;
    g->hro.push_back(0);
    if (mode == CFDXG_GAUGE_ELIMINATE) {
        g->n_out = n - 1;
        for (int64_t i = 0; i < n; ++i) {
            if (i == ref) continue;
            for (uint32_t k = H.ro[i]; k < H.ro[i + 1]; ++k) {
                const int64_t j = H.co[k];
                if (j == ref) continue;
                g->hco.push_back(static_cast<uint32_t>(j < ref ? j : j - 1));
                src.push_back(static_cast<int>(k));
            }
            g->hro.push_back(static_cast<uint32_t>(g->hco.size()));
        }
    } else {
        g->n_out = n;
        colref.assign(static_cast<size_t>(n), -1);
        for (int64_t i = 0; i < n; ++i) {
            if (i == ref) {
                g->hco.push_back(static_cast<uint32_t>(ref));
                src.push_back(-1);
            } else {
                for (uint32_t k = H.ro[i]; k < H.ro[i + 1]; ++k) {
                    const int64_t j = H.co[k];
                    if (j == ref) {
                        colref[i] = static_cast<int>(k);
                        continue;
                    }
                    g->hco.push_back(static_cast<uint32_t>(j));
                    src.push_back(static_cast<int>(k));
                }
            }
            g->hro.push_back(static_cast<uint32_t>(g->hco.size()));
        }
    }
    g->nnz_out = static_cast<int64_t>(g->hco.size());
    if (g->nnz_out == 0) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "the gauged system has no entries");
    std::vector<int> iro(g->hro.begin(), g->hro.end()), ico(g->hco.begin(), g->hco.end());
    g->ro.upload(iro, ctx->stream);
    g->co.upload(ico, ctx->stream);
    g->src.upload(src, ctx->stream);
    if (!colref.empty()) g->colref.upload(colref, ctx->stream);
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = g.release();
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_gauge_apply(cfdxg_context* ctx, const cfdxg_gauge* g, const cfdxg_matrix* A, const double* rhs,
                                 int32_t mem, cfdxg_matrix** gauged, double* rhs_out) {
    if (!ctx) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    check_mem_flag(mem);
    if (!g || !A || !rhs || !gauged || !rhs_out) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "missing argument");
    if (A->n != g->n || A->nnz != g->nnz_in || A->host.ro.size() != static_cast<size_t>(g->n + 1))
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "matrix pattern differs from the gauge plan's");
    cfdxg_matrix* B = *gauged;
    std::unique_ptr<cfdxg_matrix> fresh;
    if (!B) {
        fresh = std::make_unique<cfdxg_matrix>();
        B = fresh.get();
        B->n = g->n_out;
        B->nnz = g->nnz_out;
        B->host.n = g->n_out;
        B->host.ro.assign(g->hro.begin(), g->hro.end());
        B->host.co.assign(g->hco.begin(), g->hco.end());
        B->ro.resize(static_cast<size_t>(g->n_out) + 1);
        B->co.resize(static_cast<size_t>(g->nnz_out));
        CFDXG_CUDA(cudaMemcpyAsync(B->ro.get(), g->ro.get(), sizeof(int) * (g->n_out + 1), cudaMemcpyDeviceToDevice,
                                   ctx->stream));
        CFDXG_CUDA(cudaMemcpyAsync(B->co.get(), g->co.get(), sizeof(int) * g->nnz_out, cudaMemcpyDeviceToDevice,
                                   ctx->stream));
        B->va.resize(static_cast<size_t>(g->nnz_out));
    } else if (B->n != g->n_out || B->nnz != g->nnz_out) {
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "gauged matrix does not match the gauge plan");
    }
    In<double> b(ctx, rhs, g->n, mem);
    Out<double> bo(ctx, rhs_out, g->n_out, mem);
    {
        ProfScope ps(ctx, "gauge_values", 12.0 * g->nnz_out);
        k_gauge_values<<<blocks_for(g->nnz_out, kT), kT, 0, ctx->stream>>>(g->nnz_out, g->src.get(), A->va.get(),
                                                                          B->va.get());
        check_launch(ctx);
    }
    if (g->mode == CFDXG_GAUGE_ELIMINATE) {
        k_gauge_rhs_eliminate<<<blocks_for(g->n_out, kT), kT, 0, ctx->stream>>>(
            static_cast<int>(g->n_out), static_cast<int>(g->ref), b.get(), bo.get());
    } else {
        k_gauge_rhs_identity<<<blocks_for(g->n, kT), kT, 0, ctx->stream>>>(
            static_cast<int>(g->n), static_cast<int>(g->ref), g->value, g->colref.get(), A->va.get(), b.get(),
            bo.get());
    }
    check_launch(ctx);
    bo.finish();
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    B->host_values_valid = false;
    if (fresh) *gauged = fresh.release();
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_gauge_expand(cfdxg_context* ctx, const cfdxg_gauge* g, const double* x_reduced, int32_t mem,
                                  double* x) {
    if (!ctx) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    check_mem_flag(mem);
    if (!g || !x_reduced || !x) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "missing argument");
    if (g->mode != CFDXG_GAUGE_ELIMINATE)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "only an eliminated reference cell is expanded");
    In<double> xr(ctx, x_reduced, g->n_out, mem);
    Out<double> xo(ctx, x, g->n, mem);
    k_gauge_expand<<<blocks_for(g->n, kT), kT, 0, ctx->stream>>>(static_cast<int>(g->n), static_cast<int>(g->ref),
                                                                xr.get(), xo.get());
    check_launch(ctx);
    xo.finish();
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_gauge_size(const cfdxg_gauge* g, int64_t* n_out, int64_t* nnz_out) {
    if (!g) return CFDXG_ERR_INVALID_ARGUMENT;
    if (n_out) *n_out = g->n_out;
    if (nnz_out) *nnz_out = g->nnz_out;
    return CFDXG_OK;
}

extern "C" int cfdxg_gauge_destroy(cfdxg_gauge* g) {
    delete g;
    return CFDXG_OK;
}
