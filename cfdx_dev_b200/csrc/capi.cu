// capi.cu -- C ABI: contexts, matrices, the native AMG preconditioner and the
// solve_linear_system / solve_gmres entry points.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "io.h"
#include "krylov.h"
#include "mpnn.h"
#include "plan.h"

using namespace cfdxg;

namespace {

double now_seconds() {
    using clock = std::chrono::steady_clock;
    return std::chrono::duration<double>(clock::now().time_since_epoch()).count();
}

// JacobiPreconditioner (core/linalg/preconditioner.h:60-90): inverse of the first
// diagonal entry of each row.
__global__ void k_first_diag_inverse(int n, const int* ro, const int* co, const double* va, double* inv, int* status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = ro[i]; k < ro[i + 1]; ++k)
        if (co[k] == i) {
            const double v = 1.0 / va[k];
            if (!isfinite(v)) atomicOr(status, kStatusNonFinite);
            inv[i] = v;
            return;
        }
    atomicOr(status, kStatusNonFinite);
}

// The solver's own diagonal (cg_solver.h:171-189, no preconditioner object):
// the first diagonal entry of each row, which must be positive and finite.
__global__ void k_first_diag_positive(int n, const int* ro, const int* co, const double* va, double* d,
                                      int* status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = 0.0;
    for (int k = ro[i]; k < ro[i + 1]; ++k)
        if (co[k] == i) {
            v = va[k];
            break;
        }
    d[i] = v;
    if (!(v > 0.0) || !isfinite(v)) atomicOr(status, kStatusNonFinite);
}

// z = r / d (cg_solver.h:212)
__global__ void k_div_diag(int n, const double* d, const double* r, double* z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) z[i] = r[i] / d[i];
}

__global__ void k_scale(int n, const double* a, const double* b, double* out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = a[i] * b[i];
}

// max |a_k| over the stored values (diagnose_matrix max_abs_value); a
// non-finite value makes the slot NaN.
__global__ void k_absmax_values(int64_t nnz, const double* va, unsigned long long* bits) {
    double m = 0.0;
    for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < nnz; k += int64_t(gridDim.x) * blockDim.x)
        m = fmax(m, fabs(va[k]));
    // non-negative doubles order like their bit patterns
    atomicMax(bits, static_cast<unsigned long long>(__double_as_longlong(m)));
}

// measure_matrix_characteristics (core/linalg/matrix_diagnostics.h:317-355):
// bit 1 -- some |a_ij - a_ji| > 1e-12 max(1, max|a|) (a_ji = 0 when absent);
// bit 2 -- a row whose diagonal (sum of its diagonal entries) is missing,
// non-positive or not finite.
__global__ void k_cg_gate(int n, const int* ro, const int* co, const double* va,
                          const unsigned long long* max_bits, int* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double scale = fmax(1.0, __longlong_as_double(static_cast<long long>(*max_bits)));
    const double tol = 1e-12 * scale;
    double diag = 0.0;
    bool has_diag = false;
    for (int k = ro[i]; k < ro[i + 1]; ++k) {
        const int j = co[k];
        if (j == i) {
            diag += va[k];
            has_diag = true;
        }
        double aji = 0.0;
        for (int q = ro[j]; q < ro[j + 1]; ++q)
            if (co[q] == i) aji += va[q];
        if (fabs(va[k] - aji) > tol) atomicOr(flags, 1);
    }
    if (!has_diag || !(diag > 0.0) || !isfinite(diag)) atomicOr(flags, 2);
}

__global__ void k_copy(int n, const double* a, double* b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = a[i];
}

__global__ void k_check_finite(int n, const double* a, int* status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !isfinite(a[i])) atomicOr(status, kStatusNonFinite);
}

KrylovControls controls_from(const cfdxg_request& r) {
    KrylovControls c;
    c.restart_min = r.restart_min;
    c.restart_max = r.restart_max;
    c.adaptive_restart = r.adaptive_restart != 0;
    c.residual_replacement = r.residual_replacement != 0;
    c.residual_replacement_period = r.residual_replacement_period;
    c.residual_replacement_gap_ratio = r.residual_replacement_gap_ratio;
    c.target_reduction_per_cycle = r.target_reduction_per_cycle;
    c.classical_gram_schmidt = r.orthogonalization == CFDXG_ORTHO_CGS2;
    return c;
}

void fill_report(cfdxg_report* rep, const KrylovResult& r) {
    if (!rep) return;
    rep->status = r.status;
    rep->iterations = r.iterations;
    rep->residual = r.residual;
    rep->residual_relative = r.residual_relative;
    rep->residual_replacements = r.residual_replacements;
    rep->max_true_recursive_gap = r.max_true_recursive_gap;
    rep->preconditioner_applications = r.preconditioner_applications;
}

// Fine-level sweeps; -1 selects the precision's default: V(6,6), the
// reference's Balanced policy, for the FP64 cycle; V(3,3) for the FP32 cycle
// with its sparsified coarse smoothers, which measured the same FGMRES
// iteration count as V(4,4) (13 at 64^3, 6.9 instead of 7.2 ms per solve; 16
// on the 4.2 M-cell boundary layer, 19.3 instead of 21.0 ms), where V(2,2)
// took one to two iterations more.
int resolve_sweeps(int32_t v, int32_t precision) {
    return v >= 0 ? v : (precision == CFDXG_PRECISION_FP32_VCYCLE ? 3 : 6);
}

void amg_setup_impl(cfdxg_context* ctx, cfdxg_amg* amg, cfdxg_matrix* A) {
    const double t0 = now_seconds();
    matrix_sync_host_values(ctx, A);
    AmgOptions o;
    o.omega = amg->opts.omega;
    o.pre = resolve_sweeps(amg->opts.pre_sweeps, amg->opts.precision);
    o.post = resolve_sweeps(amg->opts.post_sweeps, amg->opts.precision);
    o.coarse_pre = amg->opts.coarse_pre_sweeps;
    o.coarse_post = amg->opts.coarse_post_sweeps;
    o.strength_threshold = amg->opts.strength_threshold;
    o.max_levels = amg->opts.max_levels;
    o.require_smoother_certificate = amg->opts.require_smoother_certificate != 0;
    o.constant_null_space = amg->opts.constant_null_space != 0;
    AmgHierarchy staged;
    std::string err;
    // the C/F splitting and interpolation on the host, the Galerkin products on the device
    DeviceGalerkin galerkin(ctx, A);
    const GalerkinHook hook = [&galerkin](int l, const HostCsr& a, const AmgLevel& p, int64_t nc, HostCsr& c) {
        return galerkin(l, a, p, nc, c);
    };
    if (!amg_setup(A->host, o, staged, err, &hook)) {
        amg->error = "native AMG hierarchy construction failed: " + err;
        throw Error(CFDXG_ERR_SETUP, amg->error);
    }
    std::unique_ptr<DevRefresh> refresh = galerkin.take(static_cast<int>(staged.levels.size()));
    const double t_hierarchy = now_seconds();
    std::unique_ptr<DevHierarchy<double>> d64;
    std::unique_ptr<DevHierarchy<float>> d32;
    UploadOptions up;
    up.reference_order = amg->opts.reference_order != 0;
    up.narrow_columns = amg->opts.narrow_columns != 0;
    up.constant_null_space = amg->opts.constant_null_space != 0;
    if (amg->opts.precision == CFDXG_PRECISION_FP32_VCYCLE) {
        up.coarse_dense_limit = amg->opts.coarse_dense_limit;
        up.half_values = amg->opts.half_values != 0;
        up.dense_fp64 = amg->opts.dense_fp64 != 0;
        up.coarse_drop_tolerance = amg->opts.coarse_drop_tolerance;
        d32 = upload_hierarchy<float>(ctx, staged, up, refresh.get());
    } else {
        d64 = upload_hierarchy<double>(ctx, staged, up, refresh.get());
    }
    if (std::getenv("CFDXG_SETUP_PROFILE"))
        std::fprintf(stderr, "[cfdxg setup] hierarchy %.3fs, device upload %.3fs\n", t_hierarchy - t0,
                     now_seconds() - t_hierarchy);
    // commit only after every stage succeeded (hypre_amg.cpp:163-236 is transactional)
    amg->host = std::move(staged);
    amg->d64 = std::move(d64);
    amg->d32 = std::move(d32);
    amg->refresh = std::move(refresh);
    amg->host_values_stale = false;
    amg->ctx = ctx;
    amg->ready = true;
    amg->error.clear();
    amg->setup_seconds = now_seconds() - t0;
}

}  // namespace

void cfdxg::amg_apply_device(cfdxg_context* ctx, cfdxg_amg* amg, const double* r, double* z) {
    if (amg->d32) vcycle_apply<float>(ctx, *amg->d32, r, z);
    else vcycle_apply<double>(ctx, *amg->d64, r, z);
    ++amg->applications;
}

// ---------------------------------------------------------------- context
extern "C" int cfdxg_context_create(int32_t device, cfdxg_context** out) {
    if (!out) return CFDXG_ERR_INVALID_ARGUMENT;
    auto* ctx = new (std::nothrow) cfdxg_context();
    if (!ctx) return CFDXG_ERR_OUT_OF_MEMORY;
    try {
        CFDXG_CUDA(cudaSetDevice(device));
        ctx->device = device;
        CFDXG_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        CFDXG_CUDA(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device));
        CFDXG_CUDA(cudaMalloc(&ctx->scratch.partial, sizeof(double) * kMaxReduceBlocks * 4));
        CFDXG_CUDA(cudaMalloc(&ctx->scratch.ticket, sizeof(unsigned) * 8));
        CFDXG_CUDA(cudaMemset(ctx->scratch.ticket, 0, sizeof(unsigned) * 8));
        CFDXG_CUDA(cudaMalloc(&ctx->scratch.scalars, sizeof(double) * 4096));
        CFDXG_CUDA(cudaMemset(ctx->scratch.scalars, 0, sizeof(double) * 4096));
        CFDXG_CUDA(cudaMalloc(&ctx->scratch.status, sizeof(int)));
        CFDXG_CUDA(cudaMemset(ctx->scratch.status, 0, sizeof(int)));
        CFDXG_CUDA(cudaMallocHost(&ctx->scratch.host_scalars, sizeof(double) * 4096));
        CFDXG_CUDA(cudaMallocHost(&ctx->scratch.host_status, sizeof(int)));
    } catch (const Error& e) {
        const int code = e.code;
        cfdxg_context_destroy(ctx);
        return code;
    }
    *out = ctx;
    return CFDXG_OK;
}

extern "C" int cfdxg_context_destroy(cfdxg_context* ctx) {
    if (!ctx) return CFDXG_OK;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    ctx->krylov_workspace.reset();
    for (auto& e : ctx->staging.entries) if (e.ptr) cudaFree(e.ptr);
    for (auto e : ctx->prof.pool) cudaEventDestroy(e);
    for (auto& pe : ctx->prof.pending) { cudaEventDestroy(pe.a); cudaEventDestroy(pe.b); }
    if (ctx->scratch.partial) cudaFree(ctx->scratch.partial);
    if (ctx->scratch.ticket) cudaFree(ctx->scratch.ticket);
    if (ctx->scratch.scalars) cudaFree(ctx->scratch.scalars);
    if (ctx->scratch.status) cudaFree(ctx->scratch.status);
    if (ctx->scratch.host_scalars) cudaFreeHost(ctx->scratch.host_scalars);
    if (ctx->scratch.host_status) cudaFreeHost(ctx->scratch.host_status);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return CFDXG_OK;
}

extern "C" const char* cfdxg_last_error(const cfdxg_context* ctx) { return ctx ? ctx->error.c_str() : "null context"; }
extern "C" int64_t cfdxg_kernel_launches(const cfdxg_context* ctx) { return ctx ? ctx->launches : 0; }
extern "C" void* cfdxg_context_stream(const cfdxg_context* ctx) {
    return ctx ? static_cast<void*>(ctx->stream) : nullptr;
}

extern "C" int cfdxg_profile_enable(cfdxg_context* ctx, int32_t on) {
    if (!ctx) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    prof_flush(ctx);
    ctx->prof.stats.clear();
    ctx->prof.on = on != 0;
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_profile_read(cfdxg_context* ctx, cfdxg_kernel_profile* out, int32_t max_entries,
                                  int32_t* count) {
    if (!ctx) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    prof_flush(ctx);
    const int32_t n = static_cast<int32_t>(ctx->prof.stats.size());
    if (count) *count = n;
    for (int32_t k = 0; k < n && k < max_entries && out; ++k) {
        std::memset(out[k].name, 0, sizeof(out[k].name));
        std::strncpy(out[k].name, ctx->prof.stats[k].name.c_str(), sizeof(out[k].name) - 1);
        out[k].launches = ctx->prof.stats[k].launches;
        out[k].total_ms = ctx->prof.stats[k].ms;
        out[k].bytes = ctx->prof.stats[k].bytes;
    }
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_synchronize(cfdxg_context* ctx) {
    if (!ctx) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

// ---------------------------------------------------------------- matrices
extern "C" int cfdxg_matrix_create(cfdxg_context* ctx, int64_t n, const int64_t* ro, const int64_t* co,
                                   const double* va, int32_t mem, cfdxg_matrix** out) {
    if (!ctx) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    check_mem_flag(mem);
    if (!out || n <= 0 || !ro || !co || !va) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "invalid matrix arguments");
    if (n > INT32_MAX / 2) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "matrix too large for 32-bit indices");
    auto A = std::make_unique<cfdxg_matrix>();
    A->n = n;
    std::vector<int64_t> hro(n + 1);
    if (mem == CFDXG_MEM_DEVICE) CFDXG_CUDA(cudaMemcpy(hro.data(), ro, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost));
    else std::memcpy(hro.data(), ro, sizeof(int64_t) * (n + 1));
    const int64_t nnz = hro[n];
    if (hro[0] != 0 || nnz <= 0 || nnz > INT32_MAX) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "invalid row offsets");
    std::vector<int64_t> hco(nnz);
    std::vector<double> hva(nnz);
    if (mem == CFDXG_MEM_DEVICE) {
        CFDXG_CUDA(cudaMemcpy(hco.data(), co, sizeof(int64_t) * nnz, cudaMemcpyDeviceToHost));
        CFDXG_CUDA(cudaMemcpy(hva.data(), va, sizeof(double) * nnz, cudaMemcpyDeviceToHost));
    } else {
        std::memcpy(hco.data(), co, sizeof(int64_t) * nnz);
        std::memcpy(hva.data(), va, sizeof(double) * nnz);
    }
    // SparseMatrix::from_sorted_csr validation (sparse_matrix.h:136-163)
    A->host.n = n;
    A->host.ro.resize(n + 1);
    A->host.co.resize(nnz);
    for (int64_t i = 0; i < n; ++i) {
        if (hro[i] > hro[i + 1] || hro[i + 1] > nnz) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "invalid offsets");
        for (int64_t k = hro[i]; k < hro[i + 1]; ++k) {
            if (hco[k] < 0 || hco[k] >= n || !std::isfinite(hva[k]) || (k > hro[i] && hco[k - 1] >= hco[k]))
                throw Error(CFDXG_ERR_INVALID_ARGUMENT, "invalid CSR row");
        }
    }
    std::vector<int> iro(n + 1), ico(nnz);
    for (int64_t i = 0; i <= n; ++i) { iro[i] = static_cast<int>(hro[i]); A->host.ro[i] = static_cast<uint32_t>(hro[i]); }
    for (int64_t k = 0; k < nnz; ++k) { ico[k] = static_cast<int>(hco[k]); A->host.co[k] = static_cast<uint32_t>(hco[k]); }
    A->host.va.assign(hva.begin(), hva.end());
    A->host_values_valid = true;
    A->nnz = nnz;
    A->ro.upload(iro, ctx->stream);
    A->co.upload(ico, ctx->stream);
    A->va.upload(A->host.va.data(), A->host.va.size(), ctx->stream);
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = A.release();
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_matrix_destroy(cfdxg_matrix* A) {
    delete A;
    return CFDXG_OK;
}

extern "C" int cfdxg_matrix_size(const cfdxg_matrix* A, int64_t* n, int64_t* nnz) {
    if (!A) return CFDXG_ERR_INVALID_ARGUMENT;
    if (n) *n = A->n;
    if (nnz) *nnz = A->nnz;
    return CFDXG_OK;
}

extern "C" int cfdxg_matrix_download(cfdxg_context* ctx, const cfdxg_matrix* A, int64_t* ro, int64_t* co, double* va) {
    if (!ctx || !A) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    if (ro) for (int64_t i = 0; i <= A->n; ++i) ro[i] = A->host.ro[i];
    if (co) for (int64_t k = 0; k < A->nnz; ++k) co[k] = A->host.co[k];
    if (va) {
        A->va.download(va, ctx->stream);
        CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_matrix_spmv(cfdxg_context* ctx, const cfdxg_matrix* A, const double* x, double* y, int32_t mem) {
    if (!ctx || !A) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    check_mem_flag(mem);
    In<double> xi(ctx, x, A->n, mem);
    Out<double> yo(ctx, y, A->n, mem);
    spmv_fp64(ctx, A, xi.get(), yo.get());
    yo.finish();
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

// ---------------------------------------------------------------- AMG
extern "C" int cfdxg_amg_options_default(cfdxg_amg_options* o) {
    if (!o) return CFDXG_ERR_INVALID_ARGUMENT;
    o->omega = 0.7;
    o->pre_sweeps = -1;
    o->post_sweeps = -1;
    o->strength_threshold = 0.25;
    o->max_levels = 25;
    o->require_smoother_certificate = 0;
    o->precision = CFDXG_PRECISION_FP64;
    o->coarse_dense_limit = 6000;
    o->reference_order = 0;
    o->coarse_pre_sweeps = -1;
    o->coarse_post_sweeps = -1;
    o->narrow_columns = 1;
    o->half_values = 1;
    o->dense_fp64 = 0;
    o->constant_null_space = 0;
    o->coarse_drop_tolerance = 0.02;
    return CFDXG_OK;
}

extern "C" int cfdxg_amg_create(cfdxg_context* ctx, const cfdxg_amg_options* opts, cfdxg_amg** out) {
    if (!out) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    auto amg = std::make_unique<cfdxg_amg>();
    if (opts) amg->opts = *opts;
    else cfdxg_amg_options_default(&amg->opts);
    const auto& o = amg->opts;
    // MatrixFreeVcyclePreconditioner constructor checks (amg_preconditioner.h:64-75)
    if (!(o.omega > 0.0 && o.omega < 2.0) || !std::isfinite(o.strength_threshold) || o.strength_threshold < 0.0 ||
        o.strength_threshold > 1.0 || o.max_levels <= 0 || o.pre_sweeps < -1 || o.post_sweeps < -1 ||
        (o.precision != CFDXG_PRECISION_FP64 && o.precision != CFDXG_PRECISION_FP32_VCYCLE) ||
        !(o.coarse_drop_tolerance >= 0.0 && o.coarse_drop_tolerance < 1.0))
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "invalid AMG operator");
    *out = amg.release();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_amg_destroy(cfdxg_amg* amg) {
    delete amg;
    return CFDXG_OK;
}

extern "C" int cfdxg_amg_setup(cfdxg_context* ctx, cfdxg_amg* amg, const cfdxg_matrix* A) {
    if (!ctx || !amg) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    NvtxRange nvtx_range("cfdxg.amg_setup");
    if (!A || A->n <= 0) {
        amg->error = "AMG setup requires a non-empty, square, finalized CSR matrix";
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, amg->error);
    }
    amg_setup_impl(ctx, amg, const_cast<cfdxg_matrix*>(A));
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_amg_update_values(cfdxg_context* ctx, cfdxg_amg* amg, const cfdxg_matrix* A) {
    if (!ctx || !amg) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    NvtxRange nvtx_range("cfdxg.amg_update_values");
    if (!amg->ready || !A) {
        amg->error = "native AMG numeric update requires an existing compatible hierarchy";
        throw Error(CFDXG_ERR_NOT_READY, amg->error);
    }
    const double t0 = now_seconds();
    std::string err;
    if (amg->d64 || amg->d32) {
        // Galerkin refresh on the device, bit-identical to the host restatement
        if (!amg_refresh_device(ctx, amg, A, err)) {
            amg->error = err;
            throw Error(CFDXG_ERR_SETUP, err);
        }
    } else {
        auto* M = const_cast<cfdxg_matrix*>(A);
        matrix_sync_host_values(ctx, M);
        if (!amg_update_values(amg->host, M->host, err)) {
            amg->error = err;
            throw Error(CFDXG_ERR_SETUP, err);
        }
    }
    amg->setup_seconds = now_seconds() - t0;
    amg->error.clear();
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_amg_update_values_host(cfdxg_amg* amg, int64_t n, const int64_t* ro, const int64_t* co,
                                            const double* va) {
    if (!amg || n <= 0 || !ro || !co || !va) return CFDXG_ERR_INVALID_ARGUMENT;
    cfdxg_context* ctx = nullptr;
    CFDXG_GUARD_BEGIN
    if (!amg->ready) {
        amg->error = "native AMG numeric update requires an existing compatible hierarchy";
        throw Error(CFDXG_ERR_NOT_READY, amg->error);
    }
    if (amg->d64 || amg->d32)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "the hierarchy lives on a device: use cfdxg_amg_update_values");
    const double t0 = now_seconds();
    HostCsr A;
    A.n = n;
    const int64_t nnz = ro[n];
    if (ro[0] != 0 || nnz <= 0 || nnz > INT32_MAX) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "invalid row offsets");
    A.ro.resize(n + 1);
    A.co.resize(nnz);
    A.va.assign(va, va + nnz);
    for (int64_t i = 0; i <= n; ++i) A.ro[i] = static_cast<uint32_t>(ro[i]);
    for (int64_t k = 0; k < nnz; ++k) {
        if (co[k] < 0 || co[k] >= n) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "column out of range");
        A.co[k] = static_cast<uint32_t>(co[k]);
    }
    std::string err;
    if (!amg_update_values(amg->host, A, err)) {
        amg->error = err;
        throw Error(CFDXG_ERR_SETUP, err);
    }
    amg->setup_seconds = now_seconds() - t0;
    amg->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_amg_apply(cfdxg_context* ctx, cfdxg_amg* amg, const double* r, double* z, int32_t mem) {
    if (!ctx || !amg) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    NvtxRange nvtx_range("cfdxg.amg_apply");
    check_mem_flag(mem);
    if (!amg->ready || (!amg->d64 && !amg->d32)) {
        amg->error = "native AMG preconditioner has not been set up on the device";
        throw Error(CFDXG_ERR_NOT_READY, amg->error);
    }
    const int64_t n = amg->host.levels.front().A.n;
    In<double> rin(ctx, r, n, mem);
    Out<double> zout(ctx, z, n, mem);
    clear_status(ctx);
    k_check_finite<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(static_cast<int>(n), rin.get(), ctx->scratch.status);
    check_launch(ctx);
    amg_apply_device(ctx, amg, rin.get(), zout.get());
    zout.finish();
    if (read_status(ctx) & kStatusNonFinite) {
        amg->error = "native AMG V-cycle failed";
        throw Error(CFDXG_ERR_NONFINITE, amg->error);
    }
    amg->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_amg_setup_host(cfdxg_amg* amg, int64_t n, const int64_t* ro, const int64_t* co,
                                    const double* va) {
    if (!amg || n <= 0 || !ro || !co || !va) return CFDXG_ERR_INVALID_ARGUMENT;
    cfdxg_context* ctx = nullptr;
    CFDXG_GUARD_BEGIN
    const double t0 = now_seconds();
    HostCsr A;
    A.n = n;
    const int64_t nnz = ro[n];
    if (ro[0] != 0 || nnz <= 0 || nnz > INT32_MAX) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "invalid row offsets");
    A.ro.resize(n + 1);
    A.co.resize(nnz);
    A.va.assign(va, va + nnz);
    for (int64_t i = 0; i <= n; ++i) A.ro[i] = static_cast<uint32_t>(ro[i]);
    for (int64_t k = 0; k < nnz; ++k) {
        if (co[k] < 0 || co[k] >= n) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "column out of range");
        A.co[k] = static_cast<uint32_t>(co[k]);
    }
    AmgOptions o;
    o.omega = amg->opts.omega;
    o.pre = resolve_sweeps(amg->opts.pre_sweeps, amg->opts.precision);
    o.post = resolve_sweeps(amg->opts.post_sweeps, amg->opts.precision);
    o.coarse_pre = amg->opts.coarse_pre_sweeps;
    o.coarse_post = amg->opts.coarse_post_sweeps;
    o.strength_threshold = amg->opts.strength_threshold;
    o.max_levels = amg->opts.max_levels;
    o.require_smoother_certificate = amg->opts.require_smoother_certificate != 0;
    o.constant_null_space = amg->opts.constant_null_space != 0;
    AmgHierarchy staged;
    std::string err;
    if (!amg_setup(A, o, staged, err)) {
        amg->error = "native AMG hierarchy construction failed: " + err;
        return CFDXG_ERR_SETUP;
    }
    amg->host = std::move(staged);
    amg->d64.reset();
    amg->d32.reset();
    amg->refresh.reset();
    amg->host_values_stale = false;
    amg->ctx = nullptr;
    amg->ready = true;
    amg->error.clear();
    amg->setup_seconds = now_seconds() - t0;
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" const char* cfdxg_amg_name(const cfdxg_amg* amg) {
    if (amg && amg->opts.precision == CFDXG_PRECISION_FP32_VCYCLE) return "NativeBoomerStyleAMG-FP32Vcycle";
    return "NativeBoomerStyleAMG";
}
extern "C" const char* cfdxg_amg_last_error(const cfdxg_amg* amg) { return amg ? amg->error.c_str() : ""; }
extern "C" int32_t cfdxg_amg_num_levels(const cfdxg_amg* amg) {
    return amg && amg->ready ? static_cast<int32_t>(amg->host.levels.size()) : 0;
}
extern "C" double cfdxg_amg_omega(const cfdxg_amg* amg) { return amg && amg->ready ? amg->host.omega : 0.0; }
extern "C" double cfdxg_amg_setup_seconds(const cfdxg_amg* amg) { return amg ? amg->setup_seconds : 0.0; }

extern "C" int cfdxg_amg_level_info(const cfdxg_amg* amg, int32_t level, int64_t* n, int64_t* nnz, int64_t* p_nnz) {
    if (!amg || !amg->ready || level < 0 || level >= static_cast<int32_t>(amg->host.levels.size()))
        return CFDXG_ERR_INVALID_ARGUMENT;
    const auto& L = amg->host.levels[level];
    if (n) *n = L.A.n;
    if (nnz) *nnz = L.A.nnz();
    if (p_nnz) *p_nnz = static_cast<int64_t>(L.p_col.size());
    return CFDXG_OK;
}

extern "C" int cfdxg_amg_export_level(const cfdxg_amg* amg, int32_t level, int64_t* ro, int64_t* co, double* va,
                                      double* inv_diag, int64_t* po, int64_t* pc, double* pv, int64_t* aggregate) {
    if (!amg || !amg->ready || level < 0 || level >= static_cast<int32_t>(amg->host.levels.size()))
        return CFDXG_ERR_INVALID_ARGUMENT;
    if (amg->host_values_stale) {   // values refreshed on the device since setup
        try {
            amg_sync_host_values(amg->ctx, const_cast<cfdxg_amg*>(amg));
        } catch (const std::exception&) {
            return CFDXG_ERR_CUDA;
        }
    }
    const auto& L = amg->host.levels[level];
    if (ro) for (std::size_t i = 0; i < L.A.ro.size(); ++i) ro[i] = L.A.ro[i];
    if (co) for (std::size_t k = 0; k < L.A.co.size(); ++k) co[k] = L.A.co[k];
    if (va) std::memcpy(va, L.A.va.data(), sizeof(double) * L.A.va.size());
    if (inv_diag) std::memcpy(inv_diag, L.inv_diag.data(), sizeof(double) * L.inv_diag.size());
    if (po && !L.p_off.empty()) for (std::size_t i = 0; i < L.p_off.size(); ++i) po[i] = L.p_off[i];
    if (pc) for (std::size_t k = 0; k < L.p_col.size(); ++k) pc[k] = L.p_col[k];
    if (pv && !L.p_val.empty()) std::memcpy(pv, L.p_val.data(), sizeof(double) * L.p_val.size());
    if (aggregate) for (std::size_t i = 0; i < L.aggregate.size(); ++i) aggregate[i] = L.aggregate[i];
    return CFDXG_OK;
}

// ---------------------------------------------------------------- solves
extern "C" int cfdxg_request_default(cfdxg_request* r) {
    if (!r) return CFDXG_ERR_INVALID_ARGUMENT;
    std::memset(r, 0, sizeof(*r));
    r->krylov = CFDXG_KRYLOV_GMRES;
    r->preconditioner = CFDXG_PC_NATIVE_AMG;
    r->gmres_restart = 40;
    r->precision = CFDXG_PRECISION_FP64;
    r->restart_min = 10;
    r->restart_max = 512;
    r->adaptive_restart = 1;
    r->residual_replacement = 1;
    r->residual_replacement_period = 50;
    r->residual_replacement_gap_ratio = 10.0;
    r->target_reduction_per_cycle = 0.1;
    r->learned = nullptr;
    r->learned_applications = 1;
    r->problem = CFDXG_PROBLEM_PRESSURE_POISSON;
    return CFDXG_OK;
}

extern "C" const char* cfdxg_plan_reason(const cfdxg_context* ctx) { return ctx ? ctx->plan_reason.c_str() : ""; }

namespace {

// Runs the Krylov solve on device vectors with an optional prepared AMG, Jacobi
// inverse diagonal, and learned network.  `setup`, when given, prepares the
// preconditioner where the solver does (CG and the projected GMRES: after the
// initial-residual check); with the constant null space the solve is the
// projected one.
KrylovResult run_krylov(cfdxg_context* ctx, const cfdxg_matrix* A, cfdxg_amg* amg, const double* inv_diag,
                        const double* b, double* x, const cfdxg_request& req, int64_t max_it, double tol,
                        int64_t* learned_fallbacks, const std::function<bool()>* setup = nullptr) {
    const bool null_space = req.null_space == CFDXG_NULL_SPACE_CONSTANT;
    RightPreconditioner pc;
    const int n = static_cast<int>(A->n);
    if (req.krylov == CFDXG_KRYLOV_CG) {
        // The preconditioner objects solve_linear_system builds for CG
        // (linear_solver_dispatch.h:169-189): identity for None, Jacobi's
        // inverse diagonal, or the native AMG V-cycle.
        if (req.preconditioner == CFDXG_PC_NATIVE_AMG)
            pc = [ctx, amg](const double* v, double* z, int) {
                amg_apply_device(ctx, amg, v, z);
                return true;
            };
        else if (req.preconditioner == CFDXG_PC_JACOBI)
            pc = [ctx, inv_diag, n](const double* v, double* z, int) {
                k_scale<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(n, inv_diag, v, z);
                check_launch(ctx);
                return true;
            };
        else if (req.preconditioner == CFDXG_PC_OWN_DIAGONAL)   // inv_diag holds the diagonal itself
            pc = [ctx, inv_diag, n](const double* v, double* z, int) {
                k_div_diag<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(n, inv_diag, v, z);
                check_launch(ctx);
                return true;
            };
        else
            pc = [ctx, n](const double* v, double* z, int) {
                k_copy<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(n, v, z);
                check_launch(ctx);
                return true;
            };
        return cg_solve(ctx, A, b, x, max_it, tol, pc, setup, req.preconditioner == CFDXG_PC_OWN_DIAGONAL,
                        null_space);
    }
    // Learned stage: dropped for the rest of the solve (plain AMG fallback)
    // as soon as an iteration fails to cut the residual estimate by 10%.
    struct LearnedState {
        bool active = true;
        double last = std::numeric_limits<double>::infinity();
        int64_t fallbacks = 0;
    } state;
    IterationObserver observer = [&state](double est) {
        if (state.active && !(est < 0.9 * state.last)) state.active = false;
        state.last = est;
    };
    if (req.learned && amg) {
        const int limit = req.learned_applications;
        pc = [ctx, amg, A, &req, &state, limit](const double* v, double* z, int j) {
            auto vcycle = [ctx, amg](const double* r, double* zz) { amg_apply_device(ctx, amg, r, zz); };
            if (limit > 0 && j >= limit) {   // the cycle's later Arnoldi vectors: the V-cycle alone
                vcycle(v, z);
                return true;
            }
            if (!state.active) {
                ++state.fallbacks;
                vcycle(v, z);
                return true;
            }
            return learned_then_amg(ctx, req.learned, A, v, z, vcycle, nullptr);
        };
    } else if (amg) {
        pc = [ctx, amg](const double* v, double* z, int) {
            amg_apply_device(ctx, amg, v, z);
            return true;
        };
    } else if (inv_diag) {
        pc = [ctx, inv_diag, n](const double* v, double* z, int) {
            k_scale<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(n, inv_diag, v, z);
            check_launch(ctx);
            return true;
        };
    }
    const RightPreconditioner* p = pc ? &pc : nullptr;
    if (null_space)
        return projected_gmres_solve(ctx, A, b, x, req.gmres_restart, max_it, tol, p, controls_from(req), nullptr,
                                     setup);
    KrylovResult r = gmres_solve(ctx, A, b, x, req.gmres_restart, max_it, tol, p, controls_from(req),
                                 req.learned && amg ? &observer : nullptr);
    if (learned_fallbacks) *learned_fallbacks = state.fallbacks;
    return r;
}

void validate_request(const cfdxg_request& r) {
    if (r.gmres_restart <= 0) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "GMRES restart must be positive");
    if (r.problem < CFDXG_PROBLEM_GENERAL || r.problem > CFDXG_PROBLEM_COUPLED_PRESSURE_VELOCITY)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "unknown problem kind");
    // select_linear_solver's model checks (linear_solver_models.h:389-398)
    const bool elliptic = r.problem == CFDXG_PROBLEM_PRESSURE_POISSON || r.problem == CFDXG_PROBLEM_DIFFUSION;
    if (r.krylov == CFDXG_KRYLOV_CG && !elliptic)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "CG needs a pressure or diffusion operator");
    if (r.preconditioner == CFDXG_PC_NATIVE_AMG && !elliptic)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "native AMG is qualified for SPD elliptic problems only");
    if (r.krylov != CFDXG_KRYLOV_GMRES && r.krylov != CFDXG_KRYLOV_FGMRES && r.krylov != CFDXG_KRYLOV_CG)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "only CG, GMRES and FGMRES are provided");
    if (r.krylov == CFDXG_KRYLOV_CG && r.learned)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "the learned stage is a variable preconditioner: it needs FGMRES");
    if (r.preconditioner != CFDXG_PC_NONE && r.preconditioner != CFDXG_PC_JACOBI &&
        r.preconditioner != CFDXG_PC_NATIVE_AMG && r.preconditioner != CFDXG_PC_OWN_DIAGONAL)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "requested preconditioner model is not implemented");
    if (r.preconditioner == CFDXG_PC_OWN_DIAGONAL && r.krylov != CFDXG_KRYLOV_CG)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "the solver's own diagonal scaling is CG's");
    if (r.precision != CFDXG_PRECISION_FP64 && r.precision != CFDXG_PRECISION_FP32_VCYCLE)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "unknown precision");
    if (r.learned && r.preconditioner != CFDXG_PC_NATIVE_AMG)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "the learned preconditioner runs in front of native AMG");
    if (r.learned_applications < 0) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "learned_applications must be >= 0");
    if (r.orthogonalization != CFDXG_ORTHO_MGS2 && r.orthogonalization != CFDXG_ORTHO_CGS2)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "unknown orthogonalization");
    if (r.scaling < CFDXG_SCALING_NONE || r.scaling > CFDXG_SCALING_SYMMETRIC_DIAGONAL)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "unknown scaling model");
    // linear_solver_dispatch.h:283-297
    if (r.krylov == CFDXG_KRYLOV_CG && r.scaling != CFDXG_SCALING_NONE && r.scaling != CFDXG_SCALING_SYMMETRIC_DIAGONAL)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "CG requires symmetry-preserving scaling (symmetric_diagonal)");
    if (r.scaling != CFDXG_SCALING_NONE && r.problem == CFDXG_PROBLEM_COUPLED_PRESSURE_VELOCITY)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "scaling is provided for scalar systems only");
    // linear_solver_dispatch.h:292-295, linear_solver_models.h:415-423
    if (r.null_space != CFDXG_NULL_SPACE_NONE && r.null_space != CFDXG_NULL_SPACE_CONSTANT)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "unknown null-space model");
    if (r.null_space == CFDXG_NULL_SPACE_CONSTANT) {
        if (r.scaling != CFDXG_SCALING_NONE)
            throw Error(CFDXG_ERR_INVALID_ARGUMENT,
                        "explicit algebraic scaling is not currently combined with a projected null-space solve");
        if (!elliptic)
            throw Error(CFDXG_ERR_INVALID_ARGUMENT,
                        "constant null space is currently qualified only for pressure/diffusion problems");
        if (r.learned)
            throw Error(CFDXG_ERR_INVALID_ARGUMENT, "the learned stage is not combined with a projected null space");
    }
}

// Scaled solve (linear_solver_dispatch.h:302-328, 466-490): scale_matrix on
// the host, the scaled system solved to a tenth of the tolerance by the
// unscaled dispatch, the solution unscaled (x_i = c_i * y_i) and certified on
// the original system, whose FP64 true residual also replaces the reported
// residuals.  Rows or columns left unscaled (zero maximum) make the request
// NOT_APPLICABLE with x untouched and an infinite physical residual.
int solve_scaled(cfdxg_context* ctx, const cfdxg_matrix* A, const double* rhs, double* x, int32_t mem,
                 const cfdxg_request& req, int64_t max_iterations, double tolerance, cfdxg_report* report) {
    const int64_t n = A->n, nnz = A->nnz;
    std::vector<double> downloaded;
    const double* hv = A->host.va.data();
    if (!A->host_values_valid) {
        downloaded.resize(static_cast<size_t>(nnz));
        A->va.download(downloaded.data(), ctx->stream);
        CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
        hv = downloaded.data();
    }
    std::vector<double> b(n), x0(n), rs(n), cs(n), sv(nnz);
    const cudaMemcpyKind to_host = mem == CFDXG_MEM_DEVICE ? cudaMemcpyDeviceToHost : cudaMemcpyHostToHost;
    CFDXG_CUDA(cudaMemcpy(b.data(), rhs, sizeof(double) * n, to_host));
    CFDXG_CUDA(cudaMemcpy(x0.data(), x, sizeof(double) * n, to_host));
    int64_t zero_rows = 0, zero_cols = 0;
    scale_values(req.scaling, n, A->host.ro.data(), A->host.co.data(), hv, 0.0, rs.data(), cs.data(), sv.data(),
                 zero_rows, zero_cols);
    if (report) std::memset(report, 0, sizeof(*report));
    if (zero_rows || zero_cols) {
        ctx->error = "scaling left a zero row or column";
        if (report) {
            report->status = CFDXG_NOT_APPLICABLE;
            report->physical_residual_relative = std::numeric_limits<double>::infinity();
            report->plan_krylov = req.krylov;
            report->plan_preconditioner = req.preconditioner;
        }
        return CFDXG_NOT_APPLICABLE;
    }
    std::vector<int64_t> ro(A->host.ro.begin(), A->host.ro.end()), co(A->host.co.begin(), A->host.co.end());
    cfdxg_matrix* As = nullptr;
    int rc = cfdxg_matrix_create(ctx, n, ro.data(), co.data(), sv.data(), CFDXG_MEM_HOST, &As);
    if (rc != CFDXG_OK) return rc;
    std::unique_ptr<cfdxg_matrix, int (*)(cfdxg_matrix*)> hold(As, cfdxg_matrix_destroy);
    std::vector<double> bs(n), xs(n);
    for (int64_t i = 0; i < n; ++i) {
        bs[i] = rs[i] * b[i];
        xs[i] = x0[i] / cs[i];
    }
    cfdxg_request inner = req;
    inner.scaling = CFDXG_SCALING_NONE;
    cfdxg_report rin{};
    const double t0 = now_seconds();
    const std::string plan = ctx->plan_reason;      // the inner, explicit solve draws no plan
    rc = cfdxg_solve_linear_system(ctx, As, bs.data(), xs.data(), CFDXG_MEM_HOST, &inner, max_iterations,
                                   0.1 * tolerance, &rin);
    ctx->plan_reason = plan;
    if (rc < 0) return rc;
    std::vector<double> xr(n);
    for (int64_t i = 0; i < n; ++i) xr[i] = cs[i] * xs[i];
    // the certificate on the original system, with the homogeneous reference for b = 0
    DevBuf<double> db(n), dx(n);
    db.upload(b, ctx->stream);
    dx.upload(x0, ctx->stream);
    const double rhs_norm = device_norm2(ctx, A, db.get());
    const double homogeneous = rhs_norm == 0.0 ? device_residual_norm(ctx, A, db.get(), dx.get()) : 0.0;
    dx.upload(xr, ctx->stream);
    const double final_residual = device_residual_norm(ctx, A, db.get(), dx.get());
    const double reference = rhs_norm > 0.0 ? rhs_norm : homogeneous;
    const double physical = reference > 0.0 ? final_residual / reference
                                            : (final_residual == 0.0 ? 0.0 : std::numeric_limits<double>::infinity());
    int status = rin.status;
    if (status == CFDXG_CONVERGED && (!std::isfinite(physical) || physical > tolerance)) status = CFDXG_MAX_ITER_REACHED;
    const cudaMemcpyKind from_host = mem == CFDXG_MEM_DEVICE ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost;
    CFDXG_CUDA(cudaMemcpy(x, xr.data(), sizeof(double) * n, from_host));
    if (report) {
        *report = rin;
        report->status = status;
        report->physical_residual_relative = physical;
        report->residual_relative = physical;
        report->residual = physical * rhs_norm;
        report->solve_seconds = now_seconds() - t0 - rin.setup_seconds;
    }
    return status;
}

// CFDX_KRYLOV_DIAGNOSTICS, the reference's switch (core/linalg/krylov_diagnostics.h:25-41):
// unset or "0" is off; any other value prints one summary line per solve on stderr.
bool krylov_diagnostics() {
    static const bool on = [] {
        const char* e = std::getenv("CFDX_KRYLOV_DIAGNOSTICS");
        return e && e[0] && std::string(e) != "0";
    }();
    return on;
}

void log_solve(const char* entry, const cfdxg_request& req, const KrylovResult& r, double physical,
               const std::string& plan) {
    if (!krylov_diagnostics()) return;
    std::fprintf(stderr,
                 "KRYLOV_SUMMARY entry=%s krylov=%s preconditioner=%s precision=%d status=%d iterations=%lld "
                 "residual_relative=%.6e physical_residual_relative=%.6e replacements=%lld%s%s%s\n",
                 entry, krylov_model_name(req.krylov),
                 req.preconditioner == CFDXG_PC_OWN_DIAGONAL ? "own_diagonal"
                                                             : preconditioner_model_name(req.preconditioner),
                 req.precision, r.status, static_cast<long long>(r.iterations), r.residual_relative, physical,
                 static_cast<long long>(r.residual_replacements), plan.empty() ? "" : " plan=\"",
                 plan.c_str(), plan.empty() ? "" : "\"");
}

// measure_matrix_characteristics' symmetry and positive-diagonal test, on the device.
bool symmetric_positive_diagonal(cfdxg_context* ctx, const cfdxg_matrix* A) {
    DevBuf<unsigned long long> max_bits(1);
    DevBuf<int> flags(1);
    CFDXG_CUDA(cudaMemsetAsync(max_bits.get(), 0, sizeof(unsigned long long), ctx->stream));
    CFDXG_CUDA(cudaMemsetAsync(flags.get(), 0, sizeof(int), ctx->stream));
    const int nb = static_cast<int>(std::min<int64_t>(std::max<int64_t>(blocks_for(A->nnz, 256), 1), 148 * 8));
    k_absmax_values<<<nb, 256, 0, ctx->stream>>>(A->nnz, A->va.get(), max_bits.get());
    k_cg_gate<<<blocks_for(A->n, 256), 256, 0, ctx->stream>>>(static_cast<int>(A->n), A->ro.get(), A->co.get(),
                                                              A->va.get(), max_bits.get(), flags.get());
    check_launch(ctx);
    int h = 0;
    CFDXG_CUDA(cudaMemcpyAsync(&h, flags.get(), sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    return h == 0;
}

}  // namespace

extern "C" int cfdxg_solve_linear_system(cfdxg_context* ctx, const cfdxg_matrix* A, const double* rhs, double* x,
                                         int32_t mem, const cfdxg_request* req_in, int64_t max_iterations,
                                         double tolerance, cfdxg_report* report) {
    if (!ctx) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    NvtxRange nvtx_range("cfdxg.solve_linear_system");
    check_mem_flag(mem);
    if (!A || !rhs || !x) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "missing argument");
    cfdxg_request req;
    if (req_in) req = *req_in;
    else cfdxg_request_default(&req);
    ctx->plan_reason.clear();
    // automatic plan (linear_solver_dispatch.h:251-268): measure, then select
    bool not_provided = false;
    if (req.krylov == CFDXG_KRYLOV_AUTO || req.preconditioner == CFDXG_PC_AUTO) {
        std::vector<double> downloaded;
        const double* hv = A->host.va.data();
        if (!A->host_values_valid) {
            downloaded.resize(static_cast<size_t>(A->nnz));
            A->va.download(downloaded.data(), ctx->stream);
            CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
            hv = downloaded.data();
        }
        cfdxg_matrix_characteristics ch;
        measure_characteristics(A->n, A->host.ro.data(), A->host.co.data(), hv,
                                req.problem == CFDXG_PROBLEM_COUPLED_PRESSURE_VELOCITY, 1e-12, ch);
        if (req.krylov == CFDXG_KRYLOV_CG && !(ch.numerically_symmetric && ch.positive_diagonal)) {
            // a forced CG fails closed before any plan is drawn
            req.preconditioner = CFDXG_PC_NONE;
        } else {
            const cfdxg_plan_request pr{req.krylov, req.preconditioner, req.gmres_restart, req.null_space,
                                        req.scaling, 1.0};
            cfdxg_solver_plan plan;
            std::string why;
            if (!select_solver(req.problem, ch, pr, plan, why)) throw Error(CFDXG_ERR_INVALID_ARGUMENT, why);
            ctx->plan_reason = plan.reason;
            const bool krylov_ok = plan.krylov == CFDXG_KRYLOV_CG || plan.krylov == CFDXG_KRYLOV_GMRES ||
                                   plan.krylov == CFDXG_KRYLOV_FGMRES;
            const bool pc_ok = plan.preconditioner == CFDXG_PC_NONE || plan.preconditioner == CFDXG_PC_JACOBI ||
                               plan.preconditioner == CFDXG_PC_NATIVE_AMG;
            if (krylov_ok && pc_ok) {
                req.krylov = plan.krylov;
                req.preconditioner = plan.preconditioner;
            } else {
                not_provided = true;
                req.krylov = krylov_ok ? plan.krylov : CFDXG_KRYLOV_GMRES;
                req.preconditioner = CFDXG_PC_NONE;
            }
        }
    }
    validate_request(req);
    if (req.scaling != CFDXG_SCALING_NONE && !not_provided)
        return solve_scaled(ctx, A, rhs, x, mem, req, max_iterations, tolerance, report);
    if (report) std::memset(report, 0, sizeof(*report));
    const int64_t n = A->n;
    In<double> b(ctx, rhs, n, mem);
    Out<double> xo(ctx, x, n, mem, /*preload=*/true);
    const double t0 = now_seconds();
    // physical reference norms (linear_solver_dispatch.h:269-273)
    const double rhs_norm = device_norm2(ctx, A, b.get());
    const double homogeneous = rhs_norm == 0.0 ? device_residual_norm(ctx, A, b.get(), xo.get()) : 0.0;
    KrylovResult r;
    int64_t learned_fallbacks = 0;
    double setup_s = 0.0;
    const bool cg = req.krylov == CFDXG_KRYLOV_CG;
    if (not_provided) {
        // the plan names a model outside this path (BiCGStab, ILU0): x untouched
        r.status = CFDXG_NOT_APPLICABLE;
        ctx->error = "automatic plan not provided by this library: " + ctx->plan_reason;
    } else if (cg && !symmetric_positive_diagonal(ctx, A)) {
        // linear_solver_dispatch.h:259-267: a forced CG on a matrix that is not
        // symmetric with a positive diagonal fails closed, x untouched
        r.status = CFDXG_NOT_APPLICABLE;
        ctx->error = "CG rejected: measured matrix is not symmetric with a positive diagonal";
    } else if (cg) {
        // the preconditioner is set up inside CG, after the initial-residual
        // check (cg_solver.h:171-176); AMG keeps the smoother certificate
        cfdxg_amg amg;
        cfdxg_amg_options_default(&amg.opts);
        amg.opts.precision = req.precision;
        amg.opts.require_smoother_certificate = 1;
        amg.opts.constant_null_space = req.null_space == CFDXG_NULL_SPACE_CONSTANT;
        DevBuf<double> inv(req.preconditioner == CFDXG_PC_JACOBI || req.preconditioner == CFDXG_PC_OWN_DIAGONAL ? n : 0);
        std::function<bool()> setup = [&]() {
            if (req.preconditioner == CFDXG_PC_NATIVE_AMG) {
                try {
                    amg_setup_impl(ctx, &amg, const_cast<cfdxg_matrix*>(A));
                } catch (const Error& e) {
                    if (e.code != CFDXG_ERR_SETUP) throw;
                    ctx->error = amg.error;
                    setup_s = amg.setup_seconds;
                    return false;
                }
                setup_s = amg.setup_seconds;
                return true;
            }
            if (req.preconditioner == CFDXG_PC_JACOBI) {
                clear_status(ctx);
                k_first_diag_inverse<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(
                    static_cast<int>(n), A->ro.get(), A->co.get(), A->va.get(), inv.get(), ctx->scratch.status);
                check_launch(ctx);
                return read_status(ctx) == 0;
            }
            if (req.preconditioner == CFDXG_PC_OWN_DIAGONAL) {
                clear_status(ctx);
                k_first_diag_positive<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(
                    static_cast<int>(n), A->ro.get(), A->co.get(), A->va.get(), inv.get(), ctx->scratch.status);
                check_launch(ctx);
                return read_status(ctx) == 0;
            }
            return true;
        };
        r = run_krylov(ctx, A, &amg, inv.get(), b.get(), xo.get(), req, max_iterations, tolerance, nullptr, &setup);
    } else if (req.null_space == CFDXG_NULL_SPACE_CONSTANT) {
        // solve_projected_gmres (projected_gmres.h:84-150): the preconditioner
        // is set up after the null-space checks and the early exit; a failed
        // setup is NOT_APPLICABLE
        cfdxg_amg amg;
        cfdxg_amg_options_default(&amg.opts);
        amg.opts.precision = req.precision;
        amg.opts.constant_null_space = 1;
        const bool use_amg = req.preconditioner == CFDXG_PC_NATIVE_AMG;
        DevBuf<double> inv(req.preconditioner == CFDXG_PC_JACOBI ? n : 0);
        std::function<bool()> setup = [&]() {
            if (use_amg) {
                try {
                    amg_setup_impl(ctx, &amg, const_cast<cfdxg_matrix*>(A));
                } catch (const Error& e) {
                    if (e.code != CFDXG_ERR_SETUP) throw;
                    ctx->error = amg.error;
                    setup_s = amg.setup_seconds;
                    return false;
                }
                setup_s = amg.setup_seconds;
                return true;
            }
            if (req.preconditioner == CFDXG_PC_JACOBI) {
                clear_status(ctx);
                k_first_diag_inverse<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(
                    static_cast<int>(n), A->ro.get(), A->co.get(), A->va.get(), inv.get(), ctx->scratch.status);
                check_launch(ctx);
                return read_status(ctx) == 0;
            }
            return true;
        };
        r = run_krylov(ctx, A, use_amg ? &amg : nullptr, req.preconditioner == CFDXG_PC_JACOBI ? inv.get() : nullptr,
                       b.get(), xo.get(), req, max_iterations, tolerance, nullptr, &setup);
    } else if (req.preconditioner == CFDXG_PC_NATIVE_AMG) {
        cfdxg_amg amg;
        cfdxg_amg_options_default(&amg.opts);
        amg.opts.precision = req.precision;
        bool ok = true;
        try {
            amg_setup_impl(ctx, &amg, const_cast<cfdxg_matrix*>(A));
        } catch (const Error& e) {
            if (e.code != CFDXG_ERR_SETUP) throw;
            ok = false;
            ctx->error = amg.error;   // LinearSolveReport::preconditioner_error
        }
        setup_s = amg.setup_seconds;
        if (ok) {
            if (req.learned) bind_learned_to_matrix(ctx, req.learned, A);
            r = run_krylov(ctx, A, &amg, nullptr, b.get(), xo.get(), req, max_iterations, tolerance, &learned_fallbacks);
        } else {
            r.status = CFDXG_NOT_APPLICABLE;
        }
    } else if (req.preconditioner == CFDXG_PC_JACOBI) {
        DevBuf<double> inv(n);
        clear_status(ctx);
        k_first_diag_inverse<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(static_cast<int>(n), A->ro.get(), A->co.get(),
                                                                          A->va.get(), inv.get(), ctx->scratch.status);
        check_launch(ctx);
        if (read_status(ctx)) r.status = CFDXG_NOT_APPLICABLE;
        else r = run_krylov(ctx, A, nullptr, inv.get(), b.get(), xo.get(), req, max_iterations, tolerance, nullptr);
    } else {
        r = run_krylov(ctx, A, nullptr, nullptr, b.get(), xo.get(), req, max_iterations, tolerance, nullptr);
    }
    // final FP64 physical certificate (linear_solver_dispatch.h:469-491)
    const double final_residual = device_residual_norm(ctx, A, b.get(), xo.get());
    const double reference = rhs_norm > 0.0 ? rhs_norm : homogeneous;
    const double physical = reference > 0.0 ? final_residual / reference
                                            : (final_residual == 0.0 ? 0.0 : std::numeric_limits<double>::infinity());
    if (r.status == CFDXG_CONVERGED && (!std::isfinite(physical) || physical > tolerance))
        r.status = CFDXG_MAX_ITER_REACHED;
    xo.finish();
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    const double t1 = now_seconds();
    fill_report(report, r);
    if (report) {
        report->physical_residual_relative = physical;
        report->setup_seconds = setup_s;
        report->solve_seconds = t1 - t0 - setup_s;
        report->learned_fallbacks = learned_fallbacks;
        report->plan_krylov = req.krylov;
        report->plan_preconditioner = req.preconditioner;
    }
    log_solve("solve_linear_system", req, r, physical, ctx->plan_reason);
    return r.status;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_solve_gmres(cfdxg_context* ctx, const cfdxg_matrix* A, cfdxg_amg* amg, const double* rhs,
                                 double* x, int32_t mem, const cfdxg_request* req_in, int64_t max_iterations,
                                 double tolerance, cfdxg_report* report) {
    if (!ctx) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    NvtxRange nvtx_range("cfdxg.solve_gmres");
    check_mem_flag(mem);
    if (!A || !rhs || !x) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "missing argument");
    cfdxg_request req;
    if (req_in) req = *req_in;
    else cfdxg_request_default(&req);
    validate_request(req);
    if (amg && (!amg->ready || (!amg->d64 && !amg->d32)))
        throw Error(CFDXG_ERR_NOT_READY, "native AMG preconditioner has not been set up on the device");
    if (amg && amg->host.levels.front().A.n != A->n) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "AMG size mismatch");
    // CG here takes the given hierarchy, or the identity without one
    if (req.krylov == CFDXG_KRYLOV_CG) req.preconditioner = amg ? CFDXG_PC_NATIVE_AMG : CFDXG_PC_NONE;
    if (report) std::memset(report, 0, sizeof(*report));
    const int64_t n = A->n;
    In<double> b(ctx, rhs, n, mem);
    Out<double> xo(ctx, x, n, mem, /*preload=*/true);
    const double t0 = now_seconds();
    int64_t learned_fallbacks = 0;
    if (req.learned && amg) bind_learned_to_matrix(ctx, req.learned, A);
    const KrylovResult r = run_krylov(ctx, A, amg, nullptr, b.get(), xo.get(), req, max_iterations, tolerance,
                                      &learned_fallbacks);
    xo.finish();
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    fill_report(report, r);
    if (report) {
        report->physical_residual_relative = r.residual_relative;
        report->solve_seconds = now_seconds() - t0;
        report->learned_fallbacks = learned_fallbacks;
        report->plan_krylov = req.krylov;
        report->plan_preconditioner = amg ? CFDXG_PC_NATIVE_AMG : CFDXG_PC_NONE;
    }
    log_solve("solve_gmres", req, r, r.residual_relative, std::string());
    return r.status;
    CFDXG_GUARD_END(ctx)
}
