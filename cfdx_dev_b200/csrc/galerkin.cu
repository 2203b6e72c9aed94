// galerkin.cu -- numeric refresh of the AMG hierarchy on the GPU.
//
// Restates MatrixFreeVcyclePreconditioner::update_values
// (core/linalg/amg_preconditioner.h:245-314) for an unchanged fine pattern:
// the Galerkin products of GalerkinCSRProduct::accumulate /
// numeric_into_existing (core/linalg/galerkin_csr_product.h:183-212), the
// inverse diagonals of build_diagonal (:1401-1421) and the damping certificate
// of compute_stable_smoother_omega (:1362-1399), with every value formed in the
// reference's order so the refreshed hierarchy is bit-identical to the host
// refresh (this file is compiled without FMA contraction):
//
//   AP entry (i, c):   sum over A's row i in CSR order, then P's row in order,
//                      of a_ik * p_kc            (one warp per row of AP)
//   C entry (c, d):    sum over P^T's row c (fine rows in increasing order),
//                      then AP's row in order, of p_ic * ap_id
//                                                (one warp per row of C)
//   pruning:           entries with |v| <= 1e-30 are dropped; the kept set must
//                      equal the existing coarse pattern, else the refresh fails
//   damping:           per row the normalised Gershgorin sum in CSR order, the
//                      level bound its maximum (order-free), omega from the host
//
// The symbolic plans built at setup (AP and P^T A P graphs, P^T adjacency) are
// uploaded once, at the first refresh.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

#include "objects.h"

namespace cfdxg {
namespace {

constexpr int kT = 256;
constexpr int kRefreshPattern = 1 << 4;   // pruned graph changed
constexpr int kRefreshInvalid = 1 << 5;   // non-finite value, zero diagonal or bad plan entry

__device__ __forceinline__ int find_col(const int* __restrict__ col, int b, int e, int key) {
    while (b < e) {
        const int m = (b + e) >> 1;
        const int v = col[m];
        if (v == key) return m;
        if (v < key) b = m + 1;
        else e = m;
    }
    return -1;
}

// Both Galerkin products run one warp per output row.  The row's
// contributions form an ordered stream -- for AP row i the pairs (k, q) of A's
// row i in CSR order and, inside each, P's row co[k] in order; for C row c the
// pairs (t, p) of P^T's row c (fine rows increasing) and, inside each, AP's
// row t_row[t] in order.  Lanes evaluate 32 consecutive contributions at a
// time (product and target entry), then, slot by slot in stream order, the
// lane that owns the target entry (position mod 32) adds it.  Every entry
// therefore receives its contributions in exactly the order of the reference's
// row-wise accumulation, and the sum is bit-identical to it.
constexpr int kWarpRows = 8;   // warps per block

// Exclusive scan over the warp of v (lane order); returns the total in *total.
__device__ __forceinline__ int warp_exclusive_scan(int v, int lane, int* total) {
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    *total = __shfl_sync(0xffffffffu, x, 31);
    return x - v;
}

// Adds the 32 evaluated contributions (value, target position; pos < 0: none)
// in slot order, each by the lane owning its target.
__device__ __forceinline__ void ordered_add(double value, int pos, int lane, double* __restrict__ out) {
#pragma unroll 4
    for (int slot = 0; slot < 32; ++slot) {
        const double v = __shfl_sync(0xffffffffu, value, slot);
        const int p = __shfl_sync(0xffffffffu, pos, slot);
        if (p >= 0 && (p & 31) == lane) out[p] = out[p] + v;
    }
}

// AP = A P (galerkin_csr_product.h accumulate, first product)
__global__ void __launch_bounds__(32 * kWarpRows) k_ap_rows(int n, const int* __restrict__ ro,
                                                            const int* __restrict__ co,
                                                            const double* __restrict__ va,
                                                            const int* __restrict__ p_off,
                                                            const int* __restrict__ p_col,
                                                            const double* __restrict__ p_val,
                                                            const int* __restrict__ ap_off,
                                                            const int* __restrict__ ap_col,
                                                            double* __restrict__ ap, int* status) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * kWarpRows;
    for (int i = blockIdx.x * kWarpRows + (threadIdx.x >> 5); i < n; i += warps) {
        const int b = ap_off[i], e = ap_off[i + 1];
        for (int p = b + lane; p < e; p += 32) ap[p] = 0.0;
        __syncwarp();
        for (int kb = ro[i]; kb < ro[i + 1]; kb += 32) {
            const int k = kb + lane;
            int len = 0, qb = 0;
            double a = 0.0;
            if (k < ro[i + 1]) {
                const int j = co[k];
                a = va[k];
                qb = p_off[j];
                len = p_off[j + 1] - qb;
            }
            int total;
            const int start = warp_exclusive_scan(len, lane, &total);
            for (int s0 = 0; s0 < total; s0 += 32) {
                const int s = s0 + lane;
                double value = 0.0;
                int pos = -1;
                // the entry k whose segment holds s: the last lane with a
                // non-empty segment starting at or before s (warp-wide loop)
                int own = 0;
                for (int l = 0; l < 32; ++l) {
                    const int st = __shfl_sync(0xffffffffu, start, l);
                    const int ln = __shfl_sync(0xffffffffu, len, l);
                    if (ln > 0 && st <= s) own = l;
                }
                const double a_own = __shfl_sync(0xffffffffu, a, own);
                const int qb_own = __shfl_sync(0xffffffffu, qb, own);
                const int st_own = __shfl_sync(0xffffffffu, start, own);
                if (s < total) {
                    const int q = qb_own + (s - st_own);
                    const double w = p_val[q];
                    if (!isfinite(w)) atomicOr(status, kRefreshInvalid);
                    pos = find_col(ap_col, b, e, p_col[q]);
                    if (pos < 0) atomicOr(status, kRefreshInvalid);
                    value = a_own * w;
                }
                ordered_add(value, pos, lane, ap);
            }
        }
    }
}

// C = P^T (AP) (accumulate, second product)
__global__ void __launch_bounds__(32 * kWarpRows) k_c_rows(int nc, const int* __restrict__ t_off,
                                                           const int* __restrict__ t_row,
                                                           const int* __restrict__ t_pos,
                                                           const int* __restrict__ p_off,
                                                           const double* __restrict__ p_val,
                                                           const int* __restrict__ ap_off,
                                                           const int* __restrict__ ap_col,
                                                           const double* __restrict__ ap,
                                                           const int* __restrict__ c_off,
                                                           const int* __restrict__ c_col,
                                                           double* __restrict__ cv, int* status) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * kWarpRows;
    for (int c = blockIdx.x * kWarpRows + (threadIdx.x >> 5); c < nc; c += warps) {
        const int b = c_off[c], e = c_off[c + 1];
        for (int p = b + lane; p < e; p += 32) cv[p] = 0.0;
        __syncwarp();
        for (int tb = t_off[c]; tb < t_off[c + 1]; tb += 32) {
            const int t = tb + lane;
            int len = 0, pb = 0;
            double weight = 0.0;
            if (t < t_off[c + 1]) {
                const int i = t_row[t];
                weight = p_val[p_off[i] + t_pos[t]];
                pb = ap_off[i];
                len = ap_off[i + 1] - pb;
            }
            int total;
            const int start = warp_exclusive_scan(len, lane, &total);
            for (int s0 = 0; s0 < total; s0 += 32) {
                const int s = s0 + lane;
                int own = 0;
                for (int l = 0; l < 32; ++l) {
                    const int st = __shfl_sync(0xffffffffu, start, l);
                    const int ln = __shfl_sync(0xffffffffu, len, l);
                    if (ln > 0 && st <= s) own = l;
                }
                const double w_own = __shfl_sync(0xffffffffu, weight, own);
                const int pb_own = __shfl_sync(0xffffffffu, pb, own);
                const int st_own = __shfl_sync(0xffffffffu, start, own);
                double value = 0.0;
                int pos = -1;
                if (s < total) {
                    const int p = pb_own + (s - st_own);
                    pos = find_col(c_col, b, e, ap_col[p]);
                    if (pos < 0) atomicOr(status, kRefreshInvalid);
                    value = w_own * ap[p];
                }
                ordered_add(value, pos, lane, cv);
            }
        }
    }
}

// numeric_into_existing: keep |v| > 1e-30 at the existing positions; the kept
// set must be exactly the existing pattern
__global__ void k_prune_into(int64_t entries, const double* __restrict__ cv, const int* __restrict__ keep_pos,
                             double* __restrict__ out, int* status) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= entries) return;
    const double v = cv[p];
    const bool keep = fabs(v) > 1e-30;
    const int pos = keep_pos[p];
    if (keep != (pos >= 0)) { atomicOr(status, kRefreshPattern); return; }
    if (keep) out[pos] = v;
}

// build_diagonal (amg_preconditioner.h:1401-1421) and the finite-value check of matrix_is_valid
__global__ void k_inverse_diagonal(int n, const int* __restrict__ ro, const int* __restrict__ co,
                                   const double* __restrict__ va, double* __restrict__ inv, int* status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double diagonal = 0.0;
    for (int k = ro[i]; k < ro[i + 1]; ++k) {
        if (!isfinite(va[k])) { atomicOr(status, kRefreshInvalid); return; }
        if (co[k] == i) diagonal += va[k];
    }
    if (!isfinite(diagonal) || fabs(diagonal) <= 1e-30) { atomicOr(status, kRefreshInvalid); return; }
    const double r = 1.0 / diagonal;
    if (!isfinite(r)) { atomicOr(status, kRefreshInvalid); return; }
    inv[i] = r;
}

// normalized_gershgorin_upper_bound (amg_preconditioner.h:1322-1347): the
// row sums in CSR order, their maximum (order-free) into *bound.  Non-positive
// or non-finite data make the bound +inf, as on the host.
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
    // non-negative doubles order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long*>(addr), static_cast<unsigned long long>(__double_as_longlong(v)));
}

__global__ void k_gershgorin(int n, const int* __restrict__ ro, const int* __restrict__ co,
                             const double* __restrict__ va, const double* __restrict__ inv, double* bound) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    const double ii = inv[i];
    if (!(ii > 0.0) || !isfinite(ii)) { atomic_max_nonneg(bound, inf); return; }
    const double di = 1.0 / ii;
    if (!(di > 0.0) || !isfinite(di)) { atomic_max_nonneg(bound, inf); return; }
    double row_sum = 0.0;
    for (int k = ro[i]; k < ro[i + 1]; ++k) {
        const double ij = inv[co[k]];
        const double dj = 1.0 / ij;
        if (!(ij > 0.0) || !isfinite(ij) || !(dj > 0.0) || !isfinite(dj)) { atomic_max_nonneg(bound, inf); return; }
        const double scale = sqrt(di) * sqrt(dj);
        if (!(scale > 0.0) || !isfinite(scale)) { atomic_max_nonneg(bound, inf); return; }
        row_sum += fabs(va[k]) / scale;
    }
    if (!isfinite(row_sum)) { atomic_max_nonneg(bound, inf); return; }
    atomic_max_nonneg(bound, row_sum);
}

std::vector<int> as_int(const std::vector<uint32_t>& v) { return std::vector<int>(v.begin(), v.end()); }

void build_refresh(cfdxg_context* ctx, cfdxg_amg* amg) {
    const AmgHierarchy& h = amg->host;
    auto R = std::make_unique<DevRefresh>();
    const std::size_t nl = h.levels.size();
    R->L.resize(nl);
    cudaStream_t s = ctx->stream;
    for (std::size_t l = 0; l < nl; ++l) {
        const AmgLevel& H = h.levels[l];
        DevRefreshLevel& D = R->L[l];
        D.n = static_cast<int>(H.A.n);
        D.nnz = H.A.nnz();
        D.ro.upload(as_int(H.A.ro), s);
        D.co.upload(as_int(H.A.co), s);
        D.va.resize(static_cast<std::size_t>(D.nnz));
        D.inv_diag.resize(static_cast<std::size_t>(D.n));
        if (l + 1 < nl) {
            const GalerkinPlan& P = H.plan;
            D.n_coarse = static_cast<int>(P.n_coarse);
            D.p_off.upload(as_int(H.p_off), s);
            D.p_col.upload(as_int(H.p_col), s);
            D.p_val.upload(H.p_val, s);
            D.ap_off.upload(as_int(P.ap_off), s);
            D.ap_col.upload(as_int(P.ap_col), s);
            D.c_off.upload(as_int(P.c_off), s);
            D.c_col.upload(as_int(P.c_col), s);
            D.t_off.upload(as_int(P.t_off), s);
            D.t_row.upload(as_int(P.t_row), s);
            D.t_pos.upload(as_int(P.t_pos), s);
            // position of each symbolic coarse entry in the existing (pruned) pattern
            const HostCsr& C = h.levels[l + 1].A;
            std::vector<int> keep(P.c_col.size(), -1);
            for (int64_t c = 0; c < static_cast<int64_t>(P.n_coarse); ++c) {
                uint32_t cursor = C.ro[c];
                for (uint32_t p = P.c_off[c]; p < P.c_off[c + 1]; ++p)
                    if (cursor < C.ro[c + 1] && C.co[cursor] == P.c_col[p]) keep[p] = static_cast<int>(cursor++);
            }
            D.keep_pos.upload(keep, s);

            D.ap.resize(P.ap_col.size());
            D.cv.resize(P.c_col.size());
        }
        CFDXG_CUDA(cudaStreamSynchronize(s));   // host staging vectors are released per level
    }
    R->bounds.resize(nl);
    amg->refresh = std::move(R);
}

// has_constant_null_space (amg_preconditioner.h:1289-1308) on the device:
// each row's sum and absolute sum in CSR order (one thread per row), then the
// largest |row sum| and absolute row sum per block (maxima are order-free).
__global__ void k_row_sum_bounds(int n, const int* __restrict__ ro, const double* __restrict__ va,
                                 double* __restrict__ partial) {
    __shared__ double sm[32];
    double residual = 0.0, scale = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double sum = 0.0, norm = 0.0;
        for (int k = ro[i]; k < ro[i + 1]; ++k) {
            sum += va[k];
            norm += fabs(va[k]);
        }
        scale = fmax(scale, norm);
        residual = fmax(residual, fabs(sum));
    }
    residual = block_max(residual, sm);
    scale = block_max(scale, sm);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = residual;
        partial[2 * blockIdx.x + 1] = scale;
    }
}

bool device_has_constant_null_space(cfdxg_context* ctx, const cfdxg_matrix* A) {
    const int nb = std::max(1, std::min(blocks_for(A->n, kT), 148 * 4));
    DevBuf<double> partial(2 * static_cast<std::size_t>(nb));
    k_row_sum_bounds<<<nb, kT, 0, ctx->stream>>>(static_cast<int>(A->n), A->ro.get(), A->va.get(), partial.get());
    check_launch(ctx);
    std::vector<double> h(2 * static_cast<std::size_t>(nb));
    partial.download(h.data(), ctx->stream);
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    double residual = 0.0, scale = 0.0;
    for (int b = 0; b < nb; ++b) {
        residual = std::max(residual, h[2 * b]);
        scale = std::max(scale, h[2 * b + 1]);
    }
    const double tolerance = 256.0 * std::numeric_limits<double>::epsilon() * std::max(1.0, scale);
    return std::isfinite(residual) && residual <= tolerance;
}

}  // namespace

bool amg_refresh_device(cfdxg_context* ctx, cfdxg_amg* amg, const cfdxg_matrix* A, std::string& error) {
    AmgHierarchy& h = amg->host;
    error.clear();
    if (h.levels.empty() || A->n != h.levels.front().A.n || A->host.ro != h.levels.front().A.ro ||
        A->host.co != h.levels.front().A.co) {
        error = "native AMG numeric update requires an unchanged CSR pattern";
        return false;
    }
    if (h.options.constant_null_space && !device_has_constant_null_space(ctx, A)) {
        error = "native AMG numeric update: the operator no longer has the constant null space";
        return false;
    }
    if (!amg->refresh) build_refresh(ctx, amg);
    DevRefresh& R = *amg->refresh;
    cudaStream_t s = ctx->stream;
    const std::size_t nl = R.L.size();
    clear_status(ctx);
    int* st = ctx->scratch.status;
    // staged: level values land in R (the device hierarchies are untouched until commit)
    CFDXG_CUDA(cudaMemcpyAsync(R.L[0].va.get(), A->va.get(), sizeof(double) * A->nnz, cudaMemcpyDeviceToDevice, s));
    for (std::size_t l = 0; l < nl; ++l) {
        DevRefreshLevel& L = R.L[l];
        if (l > 0) {
            DevRefreshLevel& F = R.L[l - 1];
            {
                ProfScope ps(ctx, "refresh_galerkin_ap", 0.0);
                const int grid = std::min<int64_t>((F.n + kWarpRows - 1) / kWarpRows, 148 * 32);
                k_ap_rows<<<grid, 32 * kWarpRows, 0, s>>>(F.n, F.ro.get(), F.co.get(), F.va.get(), F.p_off.get(),
                                                          F.p_col.get(), F.p_val.get(), F.ap_off.get(),
                                                          F.ap_col.get(), F.ap.get(), st);
                check_launch(ctx);
            }
            {
                ProfScope ps(ctx, "refresh_galerkin_c", 0.0);
                const int grid = std::min<int64_t>((F.n_coarse + kWarpRows - 1) / kWarpRows, 148 * 32);
                k_c_rows<<<grid, 32 * kWarpRows, 0, s>>>(F.n_coarse, F.t_off.get(), F.t_row.get(), F.t_pos.get(),
                                                         F.p_off.get(), F.p_val.get(), F.ap_off.get(),
                                                         F.ap_col.get(), F.ap.get(), F.c_off.get(), F.c_col.get(),
                                                         F.cv.get(), st);
                check_launch(ctx);
            }
            const int64_t entries = static_cast<int64_t>(F.cv.size());
            k_prune_into<<<blocks_for(entries, kT), kT, 0, s>>>(entries, F.cv.get(), F.keep_pos.get(), L.va.get(), st);
            check_launch(ctx);
        }
        k_inverse_diagonal<<<blocks_for(L.n, kT), kT, 0, s>>>(L.n, L.ro.get(), L.co.get(), L.va.get(),
                                                              L.inv_diag.get(), st);
        check_launch(ctx);
    }
    R.bounds.zero(s);
    ProfScope ps_bounds(ctx, "refresh_gershgorin", 0.0);
    for (std::size_t l = 0; l < nl; ++l) {
        DevRefreshLevel& L = R.L[l];
        k_gershgorin<<<blocks_for(L.n, kT), kT, 0, s>>>(L.n, L.ro.get(), L.co.get(), L.va.get(), L.inv_diag.get(),
                                                        R.bounds.get() + l);
        check_launch(ctx);
    }
    std::vector<double> bounds(nl);
    R.bounds.download(bounds.data(), s);
    const int status = read_status(ctx);   // synchronises the stream
    if (status & kRefreshPattern) {
        error = "native AMG numeric update failed: the pruned coarse pattern changed";
        return false;
    }
    if (status & kRefreshInvalid) {
        error = "native AMG numeric update failed";
        return false;
    }
    // compute_stable_smoother_omega (amg_preconditioner.h:1362-1399)
    double maximum_bound = 0.0;
    bool certified = true;
    for (std::size_t l = 0; l < nl; ++l) {
        if (!std::isfinite(bounds[l]) || !(bounds[l] > 0.0)) certified = false;
        maximum_bound = std::max(maximum_bound, bounds[l]);
    }
    double omega = h.omega;
    if (certified && maximum_bound > 0.0 && std::isfinite(maximum_bound)) {
        const double w = std::min(h.options.omega, 1.8 / maximum_bound);
        if (std::isfinite(w) && w > 0.0 && w < 2.0) omega = w;
        else certified = false;
    } else {
        certified = false;
    }
    if (!certified && h.options.require_smoother_certificate) {
        error = "native AMG numeric update failed";
        return false;
    }
    // commit
    {
        ProfScope ps(ctx, "refresh_commit", 0.0);
        if (amg->d64) set_hierarchy_values_device<double>(ctx, *amg->d64, R, omega);
        if (amg->d32) set_hierarchy_values_device<float>(ctx, *amg->d32, R, omega);
    }
    h.omega = omega;
    amg->host_values_stale = true;
    return true;
}

void amg_sync_host_values(cfdxg_context* ctx, cfdxg_amg* amg) {
    if (!amg->host_values_stale || !amg->refresh) return;
    AmgHierarchy& h = amg->host;
    for (std::size_t l = 0; l < h.levels.size(); ++l) {
        h.levels[l].A.va.resize(static_cast<std::size_t>(amg->refresh->L[l].nnz));
        h.levels[l].inv_diag.resize(static_cast<std::size_t>(amg->refresh->L[l].n));
        amg->refresh->L[l].va.download(h.levels[l].A.va.data(), ctx->stream);
        amg->refresh->L[l].inv_diag.download(h.levels[l].inv_diag.data(), ctx->stream);
    }
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    amg->host_values_stale = false;
}

}  // namespace cfdxg
