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
// The symbolic plans (AP and P^T A P graphs, P^T adjacency) come from the
// first setup: built on the device by DeviceGalerkin below, or, for a
// hierarchy set up on the host, uploaded once at the first refresh.
//
// DeviceGalerkin runs the first setup's Galerkin products on the device
// (galerkin_csr_product.h:33-167 symbolic + numeric): each symbolic graph by
// expand, sort, unique -- every contribution (row, column) as a 64-bit key,
// radix-sorted, duplicates dropped, so each row's columns come out sorted and
// unique, the sets the host's marker loops produce -- the P^T adjacency by a
// stable sort of (coarse column, fine row) keys, then the numeric products of
// the refresh kernels and the pruning of |v| <= 1e-30.  The coarse operator
// is therefore the host restatement's bit for bit, and the plan stays on the
// device for later refreshes.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <climits>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <thread>

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

// The output row's columns staged in shared memory when they fit (the
// binary searches of every contribution then read shared memory); the
// position returned is global (base + index), -1 when absent.
constexpr int kStageCols = 1024;

__device__ __forceinline__ int find_staged(const int* __restrict__ col, int len, int key, int base) {
    int b = 0, e = len;
    while (b < e) {
        const int m = (b + e) >> 1;
        const int v = col[m];
        if (v == key) return base + m;
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
// time (product and target entry); lanes whose targets coincide (always from
// different source entries, since every row of P and of AP has distinct
// columns) are combined by the lowest of them, which adds their values to the
// entry in lane order -- the stream order.  Every entry therefore receives its
// contributions in exactly the order of the reference's row-wise
// accumulation, and the sum is bit-identical to it.
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

// The lane whose segment [end - len, end) holds stream index s: the number of
// lanes whose (non-decreasing) segment end is <= s, by a five-step search.
__device__ __forceinline__ int segment_owner(int end, int s) {
    int pos = 0;
#pragma unroll
    for (int step = 16; step >= 1; step >>= 1) {
        const int e = __shfl_sync(0xffffffffu, end, pos + step - 1);
        if (e <= s) pos += step;
    }
    return pos;
}

// Adds the 32 evaluated contributions (value, target position; pos < 0: none)
// to out; lanes with equal targets are added by the lowest of them in lane
// order.  stage: this warp's 32 doubles of shared memory.
__device__ __forceinline__ void ordered_add(double value, int pos, int lane, double* __restrict__ out,
                                            double* __restrict__ stage) {
    const unsigned active = __ballot_sync(0xffffffffu, pos >= 0);
    stage[lane] = value;
    __syncwarp();
    if (pos >= 0) {
        const unsigned peers = __match_any_sync(active, pos);
        if ((peers & ((1u << lane) - 1u)) == 0u) {
            double acc = out[pos];
            for (unsigned m = peers; m != 0u; m &= m - 1u) acc = acc + stage[__ffs(m) - 1];
            out[pos] = acc;
        }
    }
    __syncwarp();
}

// first index in col[b, e) (sorted) whose value is >= key
__device__ __forceinline__ int lower_bound_col(const int* __restrict__ col, int b, int e, int key) {
    while (b < e) {
        const int m = (b + e) >> 1;
        if (col[m] < key) b = m + 1;
        else e = m;
    }
    return b;
}

// Long output rows on levels with few rows are split among `splits` warps by
// their (sorted) columns: warp s of a row owns the output positions
// [b + L s / splits, b + L (s + 1) / splits) and takes from each source row
// only the entries whose column falls in its slice (a binary search in the
// sorted source row), so the entries it owns still receive every one of their
// contributions in stream order.  splits = 1 is the plain one-warp-per-row
// form.
struct RowSlice {
    int lo, hi;            // owned output positions
    int col_lo, col_hi;    // their column range [col_lo, col_hi)
};

__device__ __forceinline__ RowSlice row_slice(const int* __restrict__ col, int b, int e, int split, int splits) {
    const int len = e - b;
    RowSlice r;
    r.lo = b + static_cast<int>(static_cast<int64_t>(len) * split / splits);
    r.hi = b + static_cast<int>(static_cast<int64_t>(len) * (split + 1) / splits);
    r.col_lo = r.lo < e ? col[r.lo] : INT_MAX;
    r.col_hi = r.hi < e ? col[r.hi] : INT_MAX;
    return r;
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
                                                            double* __restrict__ ap, int splits, int* status) {
    __shared__ double stage_all[kWarpRows][32];
    __shared__ int cols_all[kWarpRows][kStageCols];
    const int lane = threadIdx.x & 31;
    double* stage = stage_all[threadIdx.x >> 5];
    int* scols = cols_all[threadIdx.x >> 5];
    const int64_t units = static_cast<int64_t>(n) * splits;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * kWarpRows;
    for (int64_t u = static_cast<int64_t>(blockIdx.x) * kWarpRows + (threadIdx.x >> 5); u < units; u += warps) {
        const int i = static_cast<int>(u / splits);
        const RowSlice sl = row_slice(ap_col, ap_off[i], ap_off[i + 1], static_cast<int>(u % splits), splits);
        const int b = sl.lo, e = sl.hi;
        const bool staged = e - b <= kStageCols;
        for (int p = b + lane; p < e; p += 32) {
            ap[p] = 0.0;
            if (staged) scols[p - b] = ap_col[p];
        }
        __syncwarp();
        if (b == e) continue;
        for (int kb = ro[i]; kb < ro[i + 1]; kb += 32) {
            const int k = kb + lane;
            int len = 0, qb = 0;
            double a = 0.0;
            if (k < ro[i + 1]) {
                const int j = co[k];
                a = va[k];
                qb = p_off[j];
                int qe = p_off[j + 1];
                if (splits > 1) {
                    qb = lower_bound_col(p_col, qb, qe, sl.col_lo);
                    qe = lower_bound_col(p_col, qb, qe, sl.col_hi);
                }
                len = qe - qb;
            }
            int total;
            const int start = warp_exclusive_scan(len, lane, &total);
            const int end = start + len;
            for (int s0 = 0; s0 < total; s0 += 32) {
                const int s = s0 + lane;
                const int own = segment_owner(end, s < total ? s : total - 1);
                const double a_own = __shfl_sync(0xffffffffu, a, own);
                const int qb_own = __shfl_sync(0xffffffffu, qb, own);
                const int st_own = __shfl_sync(0xffffffffu, start, own);
                double value = 0.0;
                int pos = -1;
                if (s < total) {
                    const int q = qb_own + (s - st_own);
                    const double w = p_val[q];
                    if (!isfinite(w)) atomicOr(status, kRefreshInvalid);
                    pos = staged ? find_staged(scols, e - b, p_col[q], b) : find_col(ap_col, b, e, p_col[q]);
                    if (pos < 0) atomicOr(status, kRefreshInvalid);
                    value = a_own * w;
                }
                ordered_add(value, pos, lane, ap, stage);
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
                                                           double* __restrict__ cv, int splits, int* status) {
    __shared__ double stage_all[kWarpRows][32];
    __shared__ int cols_all[kWarpRows][kStageCols];
    const int lane = threadIdx.x & 31;
    double* stage = stage_all[threadIdx.x >> 5];
    int* scols = cols_all[threadIdx.x >> 5];
    const int64_t units = static_cast<int64_t>(nc) * splits;
    const int64_t warps = static_cast<int64_t>(gridDim.x) * kWarpRows;
    for (int64_t u = static_cast<int64_t>(blockIdx.x) * kWarpRows + (threadIdx.x >> 5); u < units; u += warps) {
        const int c = static_cast<int>(u / splits);
        const RowSlice sl = row_slice(c_col, c_off[c], c_off[c + 1], static_cast<int>(u % splits), splits);
        const int b = sl.lo, e = sl.hi;
        const bool staged = e - b <= kStageCols;
        for (int p = b + lane; p < e; p += 32) {
            cv[p] = 0.0;
            if (staged) scols[p - b] = c_col[p];
        }
        __syncwarp();
        if (b == e) continue;
        for (int tb = t_off[c]; tb < t_off[c + 1]; tb += 32) {
            const int t = tb + lane;
            int len = 0, pb = 0;
            double weight = 0.0;
            if (t < t_off[c + 1]) {
                const int i = t_row[t];
                weight = p_val[p_off[i] + t_pos[t]];
                pb = ap_off[i];
                int pe = ap_off[i + 1];
                if (splits > 1) {
                    pb = lower_bound_col(ap_col, pb, pe, sl.col_lo);
                    pe = lower_bound_col(ap_col, pb, pe, sl.col_hi);
                }
                len = pe - pb;
            }
            int total;
            const int start = warp_exclusive_scan(len, lane, &total);
            const int end = start + len;
            for (int s0 = 0; s0 < total; s0 += 32) {
                const int s = s0 + lane;
                const int own = segment_owner(end, s < total ? s : total - 1);
                const double w_own = __shfl_sync(0xffffffffu, weight, own);
                const int pb_own = __shfl_sync(0xffffffffu, pb, own);
                const int st_own = __shfl_sync(0xffffffffu, start, own);
                double value = 0.0;
                int pos = -1;
                if (s < total) {
                    const int p = pb_own + (s - st_own);
                    pos = staged ? find_staged(scols, e - b, ap_col[p], b) : find_col(c_col, b, e, ap_col[p]);
                    if (pos < 0) atomicOr(status, kRefreshInvalid);
                    value = w_own * ap[p];
                }
                ordered_add(value, pos, lane, cv, stage);
            }
        }
    }
}

// Splits per output row: slices of at most about 256 output entries (their
// columns then always fit the shared-memory staging, and a row's stream is
// shared among warps), and enough warps to fill the GPU twice over on levels
// with few rows, each slice owning at least 32 entries.
int choose_splits(int64_t rows, int64_t entries) {
    if (rows <= 0) return 1;
    const int64_t fill = (2 * 148 * 48 + rows - 1) / rows;
    const int64_t length = entries / rows;
    const int64_t want = std::max<int64_t>(fill, length / 256);
    const int64_t cap = std::max<int64_t>(1, length / 32);
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>({want, cap, 64})));
}

int galerkin_grid(int64_t rows, int splits) {
    const int64_t units = rows * splits;
    return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>((units + kWarpRows - 1) / kWarpRows, 148 * 32)));
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

// sqrt(1 / inv_i) per row, formed once (the host forms the same value per
// entry); a non-positive or non-finite inverse diagonal or diagonal makes the
// bound +inf (every row's diagonal entry references its own inverse)
__global__ void k_sqrt_diagonal(int n, const double* __restrict__ inv, double* __restrict__ sd, double* bound) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    const double ii = inv[i];
    const double di = 1.0 / ii;
    if (!(ii > 0.0) || !isfinite(ii) || !(di > 0.0) || !isfinite(di)) {
        atomic_max_nonneg(bound, inf);
        sd[i] = 0.0;
        return;
    }
    sd[i] = sqrt(di);
}

__global__ void k_gershgorin(int n, const int* __restrict__ ro, const int* __restrict__ co,
                             const double* __restrict__ va, const double* __restrict__ sd, double* bound) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    const double si = sd[i];
    double row_sum = 0.0;
    for (int k = ro[i]; k < ro[i + 1]; ++k) {
        const double scale = si * sd[co[k]];
        if (!(scale > 0.0) || !isfinite(scale)) { atomic_max_nonneg(bound, inf); return; }
        row_sum += fabs(va[k]) / scale;
    }
    if (!isfinite(row_sum)) { atomic_max_nonneg(bound, inf); return; }
    atomic_max_nonneg(bound, row_sum);
}

// The same bound with one warp per row, for levels with long rows: the lanes
// form 32 terms at a time, and one lane adds them to the row sum in CSR
// order, so the sum is the sequential one bit for bit.
__global__ void k_gershgorin_warp(int n, const int* __restrict__ ro, const int* __restrict__ co,
                                  const double* __restrict__ va, const double* __restrict__ sd, double* bound) {
    __shared__ double terms_all[8][32];
    const int lane = threadIdx.x & 31;
    double* terms = terms_all[threadIdx.x >> 5];
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    const int warps = gridDim.x * 8;
    for (int i = blockIdx.x * 8 + (threadIdx.x >> 5); i < n; i += warps) {
        const double si = sd[i];
        double row_sum = 0.0;
        bool bad = false;
        for (int kb = ro[i]; kb < ro[i + 1]; kb += 32) {
            const int k = kb + lane;
            double term = 0.0;
            bool invalid = false;
            if (k < ro[i + 1]) {
                const double scale = si * sd[co[k]];
                invalid = !(scale > 0.0) || !isfinite(scale);
                term = fabs(va[k]) / scale;
            }
            if (__any_sync(0xffffffffu, invalid)) { bad = true; break; }
            terms[lane] = term;
            __syncwarp();
            if (lane == 0) {
                const int count = min(32, ro[i + 1] - kb);
                for (int q = 0; q < count; ++q) row_sum += terms[q];
            }
            __syncwarp();
        }
        if (lane == 0) {
            if (bad || !isfinite(row_sum)) atomic_max_nonneg(bound, inf);
            else atomic_max_nonneg(bound, row_sum);
        }
    }
}

template <class V>
std::vector<int> as_int(const V& v) { return std::vector<int>(v.begin(), v.end()); }

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

// ---- first-setup Galerkin product (expand, sort, unique) ----

// the row r with off[r] <= k < off[r + 1] (off non-decreasing, off[0] = 0)
template <class Off>
__device__ __forceinline__ int row_of(const Off* __restrict__ off, int rows, int64_t k) {
    int b = 0, e = rows;   // invariant: off[b] <= k < off[e]
    while (e - b > 1) {
        const int m = (b + e) >> 1;
        if (static_cast<int64_t>(off[m]) <= k) b = m;
        else e = m;
    }
    return b;
}

// P^T adjacency keys: (coarse column << 32 | fine row) and the entry's position in its P row
__global__ void k_pt_keys(int n, const int* __restrict__ p_off, const int* __restrict__ p_col,
                          unsigned long long* __restrict__ keys, int* __restrict__ pos) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int q = p_off[i]; q < p_off[i + 1]; ++q) {
        keys[q] = (static_cast<unsigned long long>(p_col[q]) << 32) | static_cast<unsigned>(i);
        pos[q] = q - p_off[i];
    }
}

// contributions of A's entry k to AP: the length of P's row co[k]
__global__ void k_ap_expand_len(int64_t nnz, const int* __restrict__ co, const int* __restrict__ p_off,
                                int64_t* __restrict__ len) {
    const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < nnz) len[k] = p_off[co[k] + 1] - p_off[co[k]];
}

__global__ void k_ap_expand(int64_t nnz, int n, const int* __restrict__ ro, const int* __restrict__ co,
                            const int* __restrict__ p_off, const int* __restrict__ p_col,
                            const int64_t* __restrict__ eoff, unsigned long long* __restrict__ keys) {
    const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= nnz) return;
    const unsigned long long row = static_cast<unsigned long long>(row_of(ro, n, k)) << 32;
    const int j = co[k];
    int64_t o = eoff[k];
    for (int q = p_off[j]; q < p_off[j + 1]; ++q) keys[o++] = row | static_cast<unsigned>(p_col[q]);
}

// contributions of P^T's entry t to C: the length of AP's row t_row[t]
__global__ void k_c_expand_len(int64_t tn, const int* __restrict__ t_row, const int* __restrict__ ap_off,
                               int64_t* __restrict__ len) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < tn) len[t] = ap_off[t_row[t] + 1] - ap_off[t_row[t]];
}

__global__ void k_c_expand(int64_t tn, int nc, const int* __restrict__ t_off, const int* __restrict__ t_row,
                           const int* __restrict__ ap_off, const int* __restrict__ ap_col,
                           const int64_t* __restrict__ eoff, unsigned long long* __restrict__ keys) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= tn) return;
    const unsigned long long row = static_cast<unsigned long long>(row_of(t_off, nc, t)) << 32;
    const int i = t_row[t];
    int64_t o = eoff[t];
    for (int p = ap_off[i]; p < ap_off[i + 1]; ++p) keys[o++] = row | static_cast<unsigned>(ap_col[p]);
}

// per-row counts (counts[row + 1]) and the columns of sorted unique keys
__global__ void k_key_rows(int64_t m, const unsigned long long* __restrict__ keys, int* __restrict__ counts,
                           int* __restrict__ cols) {
    const int64_t u = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (u >= m) return;
    const unsigned long long key = keys[u];
    atomicAdd(counts + (key >> 32) + 1, 1);
    cols[u] = static_cast<int>(key & 0xffffffffull);
}

// galerkin_csr_product.h:141-167 pruning: keep |v| > 1e-30
__global__ void k_prune_flags(int64_t m, const double* __restrict__ cv, int* __restrict__ flags) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p < m) flags[p] = fabs(cv[p]) > 1e-30 ? 1 : 0;
    if (p == m) flags[p] = 0;
}

__global__ void k_prune_scatter(int64_t m, const int* __restrict__ c_col, const double* __restrict__ cv,
                                const int* __restrict__ flags, const int* __restrict__ slot,
                                int* __restrict__ keep_pos, int* __restrict__ co, double* __restrict__ va) {
    const int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (p >= m) return;
    if (flags[p]) {
        const int d = slot[p];
        keep_pos[p] = d;
        co[d] = c_col[p];
        va[d] = cv[p];
    } else {
        keep_pos[p] = -1;
    }
}

__global__ void k_pruned_offsets(int nc, const int* __restrict__ c_off, const int* __restrict__ slot,
                                 int* __restrict__ ro) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c <= nc) ro[c] = slot[c_off[c]];
}

int key_bits(int64_t rows) {
    int b = 1;
    while ((int64_t{1} << b) < rows + 1) ++b;
    return 32 + b;
}

double wall_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// grow-only scratch: reallocated only when a level needs more, then with a
// quarter of headroom (the expansions grow for several levels)
template <class T>
T* grow(DevBuf<T>& b, int64_t n) {
    if (static_cast<int64_t>(b.size()) < std::max<int64_t>(n, 1)) {
        static const bool profile = std::getenv("CFDXG_SETUP_PROFILE") != nullptr;
        const double t0 = profile ? wall_seconds() : 0.0;
        b.release();
        b.resize(static_cast<std::size_t>(std::max<int64_t>(n + n / 4, 1)));
        if (profile)
            std::fprintf(stderr, "[cfdxg setup]       scratch grown to %.1f MB in %.3fs\n",
                         static_cast<double>(b.size() * sizeof(T)) / 1e6, wall_seconds() - t0);
    }
    return b.get();
}

template <class T>
void exclusive_sum(cudaStream_t s, const T* in, T* out, int64_t n, DevBuf<unsigned char>& temp) {
    std::size_t bytes = 0;
    CFDXG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s));
    CFDXG_CUDA(cub::DeviceScan::ExclusiveSum(grow(temp, static_cast<int64_t>(bytes)), bytes, in, out, n, s));
}

// sorted unique keys of keys[0, m) (bits [0, end_bit)) into out; returns their count
int64_t sort_unique(cudaStream_t s, const unsigned long long* keys, int64_t m, int end_bit,
                    DevBuf<unsigned long long>& sorted, DevBuf<unsigned long long>& out, DevBuf<int64_t>& count,
                    DevBuf<unsigned char>& temp) {
    std::size_t bytes = 0;
    unsigned long long* so = grow(sorted, m);
    CFDXG_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, bytes, keys, so, m, 0, end_bit, s));
    CFDXG_CUDA(cub::DeviceRadixSort::SortKeys(grow(temp, static_cast<int64_t>(bytes)), bytes, keys, so, m, 0,
                                              end_bit, s));
    unsigned long long* uo = grow(out, m);
    int64_t* c = grow(count, 1);
    bytes = 0;
    CFDXG_CUDA(cub::DeviceSelect::Unique(nullptr, bytes, so, uo, c, m, s));
    CFDXG_CUDA(cub::DeviceSelect::Unique(grow(temp, static_cast<int64_t>(bytes)), bytes, so, uo, c, m, s));
    int64_t h = 0;
    CFDXG_CUDA(cudaMemcpyAsync(&h, c, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CFDXG_CUDA(cudaStreamSynchronize(s));
    return h;
}

// CSR (off: rows + 1, col) of sorted unique (row << 32 | col) keys: counts[r + 1]
// = row r's length, and their inclusive sum is off
void keys_to_csr(cfdxg_context* ctx, const unsigned long long* keys, int64_t m, int rows, DevBuf<int>& off,
                 DevBuf<int>& col, DevBuf<int>& counts, DevBuf<unsigned char>& temp) {
    cudaStream_t s = ctx->stream;
    int* cnt = grow(counts, static_cast<int64_t>(rows) + 1);
    CFDXG_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (static_cast<std::size_t>(rows) + 1), s));
    col.resize(static_cast<std::size_t>(std::max<int64_t>(m, 1)));
    if (m > 0) {
        k_key_rows<<<blocks_for(m, kT), kT, 0, s>>>(m, keys, cnt, col.get());
        check_launch(ctx);
    }
    off.resize(static_cast<std::size_t>(rows) + 1);
    std::size_t bytes = 0;
    CFDXG_CUDA(cub::DeviceScan::InclusiveSum(nullptr, bytes, cnt, off.get(), rows + 1, s));
    CFDXG_CUDA(cub::DeviceScan::InclusiveSum(grow(temp, static_cast<int64_t>(bytes)), bytes, cnt, off.get(),
                                             rows + 1, s));
}

}  // namespace

DeviceGalerkin::DeviceGalerkin(cfdxg_context* ctx, const cfdxg_matrix* A)
    : ctx_(ctx), A_(A), R_(std::make_unique<DevRefresh>()) {}

DeviceGalerkin::~DeviceGalerkin() {
    for (int k = 0; k < 2; ++k) {
        if (stage_[k]) cudaFreeHost(stage_[k]);
        if (staged_[k]) cudaEventDestroy(staged_[k]);
    }
}

// memcpy split over a few host threads (the destination is first touched
// here, so its page faults are spread over the threads too)
void parallel_memcpy(char* dst, const char* src, std::size_t len) {
    constexpr std::size_t kPiece = std::size_t{4} << 20;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const std::size_t pieces = std::min<std::size_t>(std::min<unsigned>(hw, 8u), (len + kPiece - 1) / kPiece);
    if (pieces <= 1) {
        std::memcpy(dst, src, len);
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(pieces);
    for (std::size_t w = 0; w < pieces; ++w) {
        const std::size_t b = len * w / pieces, e = len * (w + 1) / pieces;
        pool.emplace_back([=] { std::memcpy(dst + b, src + b, e - b); });
    }
    for (auto& t : pool) t.join();
}

// Device-to-host copy through two fixed pinned chunks: the next chunk's
// transfer runs while the host copies the previous one out.
void DeviceGalerkin::download(const void* src, void* dst, std::size_t bytes) {
    cudaStream_t s = ctx_->stream;
    if (!stage_[0]) {
        for (int k = 0; k < 2; ++k) {
            CFDXG_CUDA(cudaHostAlloc(&stage_[k], kStageBytes, cudaHostAllocDefault));
            CFDXG_CUDA(cudaEventCreateWithFlags(&staged_[k], cudaEventDisableTiming));
        }
    }
    const char* from = static_cast<const char*>(src);
    char* to = static_cast<char*>(dst);
    const std::size_t chunks = (bytes + kStageBytes - 1) / kStageBytes;
    for (std::size_t c = 0; c <= chunks; ++c) {
        if (c < chunks) {
            const std::size_t len = std::min(kStageBytes, bytes - c * kStageBytes);
            CFDXG_CUDA(cudaMemcpyAsync(stage_[c & 1], from + c * kStageBytes, len, cudaMemcpyDeviceToHost, s));
            CFDXG_CUDA(cudaEventRecord(staged_[c & 1], s));
        }
        if (c > 0) {
            const std::size_t p = c - 1;
            const std::size_t len = std::min(kStageBytes, bytes - p * kStageBytes);
            CFDXG_CUDA(cudaEventSynchronize(staged_[p & 1]));
            parallel_memcpy(to + p * kStageBytes, static_cast<const char*>(stage_[p & 1]), len);
        }
    }
}

bool DeviceGalerkin::operator()(int level, const HostCsr& A, const AmgLevel& P, int64_t coarse_n,
                                HostCsr& coarse) {
    cudaStream_t s = ctx_->stream;
    const int64_t n = A.n, nnz = A.nnz(), pn = static_cast<int64_t>(P.p_col.size());
    if (n > std::numeric_limits<int>::max() || nnz > std::numeric_limits<int>::max() ||
        coarse_n > std::numeric_limits<int>::max() || static_cast<int64_t>(P.p_off.size()) != n + 1 ||
        static_cast<int64_t>(P.p_off[n]) != pn || static_cast<int64_t>(P.p_val.size()) != pn)
        return false;
    // galerkin_csr_product.h:52-60: every prolongation column in range, every weight finite
    for (int64_t q = 0; q < pn; ++q)
        if (P.p_col[q] >= coarse_n || !std::isfinite(P.p_val[q])) return false;
    if (static_cast<int>(R_->L.size()) < level + 2) R_->L.resize(level + 2);
    DevRefreshLevel& F = R_->L[level];
    const int nc = static_cast<int>(coarse_n);
    if (level == 0) {
        // the fine level: the device matrix itself
        F.n = static_cast<int>(n);
        F.nnz = nnz;
        F.ro.resize(n + 1);
        F.co.resize(nnz);
        F.va.resize(nnz);
        CFDXG_CUDA(cudaMemcpyAsync(F.ro.get(), A_->ro.get(), sizeof(int) * (n + 1), cudaMemcpyDeviceToDevice, s));
        CFDXG_CUDA(cudaMemcpyAsync(F.co.get(), A_->co.get(), sizeof(int) * nnz, cudaMemcpyDeviceToDevice, s));
        CFDXG_CUDA(cudaMemcpyAsync(F.va.get(), A_->va.get(), sizeof(double) * nnz, cudaMemcpyDeviceToDevice, s));
    }
    if (F.n != static_cast<int>(n) || F.nnz != nnz) return false;
    F.inv_diag.resize(static_cast<std::size_t>(n));
    F.n_coarse = nc;
    F.p_off.upload(std::vector<int>(P.p_off.begin(), P.p_off.end()), s);
    F.p_col.upload(std::vector<int>(P.p_col.begin(), P.p_col.end()), s);
    F.p_val.upload(P.p_val, s);
    clear_status(ctx_);
    int* st = ctx_->scratch.status;

    // per-phase device times with CFDXG_SETUP_PROFILE (synchronising)
    static const bool profile = std::getenv("CFDXG_SETUP_PROFILE") != nullptr;
    double tp = wall_seconds();
    auto phase = [&](const char* what) {
        if (!profile) return;
        CFDXG_CUDA(cudaStreamSynchronize(s));
        const double t = wall_seconds();
        std::fprintf(stderr, "[cfdxg setup]     device %s %.3fs\n", what, t - tp);
        tp = t;
    };
    // P^T adjacency, stable: (column, fine row) keys sorted, positions alongside
    {
        unsigned long long* keys = grow(keys_, pn);
        unsigned long long* sorted = grow(sorted_, pn);
        int* pos = grow(ints_, pn);
        F.t_pos.resize(std::max<int64_t>(pn, 1));
        k_pt_keys<<<blocks_for(n, kT), kT, 0, s>>>(static_cast<int>(n), F.p_off.get(), F.p_col.get(), keys, pos);
        check_launch(ctx_);
        std::size_t bytes = 0;
        const int end_bit = key_bits(coarse_n);
        CFDXG_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys, sorted, pos, F.t_pos.get(), pn, 0, end_bit,
                                                   s));
        CFDXG_CUDA(cub::DeviceRadixSort::SortPairs(grow(temp_, static_cast<int64_t>(bytes)), bytes, keys, sorted,
                                                   pos, F.t_pos.get(), pn, 0, end_bit, s));
        keys_to_csr(ctx_, sorted, pn, nc, F.t_off, F.t_row, counts_, temp_);   // rows: coarse columns
    }
    phase("P^T adjacency");
    // symbolic AP: every (i, p_col[q]) for k in A's row i and q in P's row co[k]
    {
        int64_t* len = grow(len_, nnz + 1);
        int64_t* eoff = grow(eoff_, nnz + 1);
        CFDXG_CUDA(cudaMemsetAsync(len + nnz, 0, sizeof(int64_t), s));
        k_ap_expand_len<<<blocks_for(nnz, kT), kT, 0, s>>>(nnz, F.co.get(), F.p_off.get(), len);
        check_launch(ctx_);
        exclusive_sum<int64_t>(s, len, eoff, nnz + 1, temp_);
        int64_t m = 0;
        CFDXG_CUDA(cudaMemcpyAsync(&m, eoff + nnz, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        CFDXG_CUDA(cudaStreamSynchronize(s));
        unsigned long long* keys = grow(keys_, m);
        k_ap_expand<<<blocks_for(nnz, kT), kT, 0, s>>>(nnz, static_cast<int>(n), F.ro.get(), F.co.get(),
                                                      F.p_off.get(), F.p_col.get(), eoff, keys);
        check_launch(ctx_);
        const int64_t u = sort_unique(s, keys, m, key_bits(n), sorted_, uniq_, count_, temp_);
        if (u > std::numeric_limits<int>::max()) return false;
        keys_to_csr(ctx_, uniq_.get(), u, static_cast<int>(n), F.ap_off, F.ap_col, counts_, temp_);
        F.ap.resize(static_cast<std::size_t>(std::max<int64_t>(u, 1)));
    }
    phase("AP graph");
    // numeric AP
    {
        const int splits = choose_splits(n, static_cast<int64_t>(F.ap.size()));
        k_ap_rows<<<galerkin_grid(n, splits), 32 * kWarpRows, 0, s>>>(
            static_cast<int>(n), F.ro.get(), F.co.get(), F.va.get(), F.p_off.get(), F.p_col.get(), F.p_val.get(),
            F.ap_off.get(), F.ap_col.get(), F.ap.get(), splits, st);
        check_launch(ctx_);
    }
    phase("AP values");
    // symbolic C = P^T (AP): every (c, ap_col[p]) for t in P^T's row c and p in AP's row t_row[t]
    int64_t cm = 0;
    {
        int64_t* len = grow(len_, pn + 1);
        int64_t* eoff = grow(eoff_, pn + 1);
        CFDXG_CUDA(cudaMemsetAsync(len + pn, 0, sizeof(int64_t), s));
        k_c_expand_len<<<blocks_for(std::max<int64_t>(pn, 1), kT), kT, 0, s>>>(pn, F.t_row.get(), F.ap_off.get(),
                                                                             len);
        check_launch(ctx_);
        exclusive_sum<int64_t>(s, len, eoff, pn + 1, temp_);
        int64_t m = 0;
        CFDXG_CUDA(cudaMemcpyAsync(&m, eoff + pn, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        CFDXG_CUDA(cudaStreamSynchronize(s));
        unsigned long long* keys = grow(keys_, m);
        k_c_expand<<<blocks_for(std::max<int64_t>(pn, 1), kT), kT, 0, s>>>(pn, nc, F.t_off.get(), F.t_row.get(),
                                                                         F.ap_off.get(), F.ap_col.get(), eoff,
                                                                         keys);
        check_launch(ctx_);
        cm = sort_unique(s, keys, m, key_bits(coarse_n), sorted_, uniq_, count_, temp_);
        if (cm > std::numeric_limits<int>::max()) return false;
        keys_to_csr(ctx_, uniq_.get(), cm, nc, F.c_off, F.c_col, counts_, temp_);
        F.cv.resize(static_cast<std::size_t>(std::max<int64_t>(cm, 1)));
    }
    phase("C graph");
    // numeric C
    {
        const int splits = choose_splits(coarse_n, cm);
        k_c_rows<<<galerkin_grid(coarse_n, splits), 32 * kWarpRows, 0, s>>>(
            nc, F.t_off.get(), F.t_row.get(), F.t_pos.get(), F.p_off.get(), F.p_val.get(), F.ap_off.get(),
            F.ap_col.get(), F.ap.get(), F.c_off.get(), F.c_col.get(), F.cv.get(), splits, st);
        check_launch(ctx_);
    }
    phase("C values");
    // pruning into the next level's CSR (device) and the refresh's keep positions
    DevRefreshLevel& C = R_->L[level + 1];
    {
        int* flags = grow(ints_, cm + 1);
        int* slot = grow(ints2_, cm + 1);
        k_prune_flags<<<blocks_for(cm + 1, kT), kT, 0, s>>>(cm, F.cv.get(), flags);
        check_launch(ctx_);
        exclusive_sum<int>(s, flags, slot, cm + 1, temp_);
        int kept = 0;
        CFDXG_CUDA(cudaMemcpyAsync(&kept, slot + cm, sizeof(int), cudaMemcpyDeviceToHost, s));
        CFDXG_CUDA(cudaStreamSynchronize(s));
        C.n = nc;
        C.nnz = kept;
        C.ro.resize(static_cast<std::size_t>(nc) + 1);
        C.co.resize(static_cast<std::size_t>(std::max(kept, 1)));
        C.va.resize(static_cast<std::size_t>(std::max(kept, 1)));
        F.keep_pos.resize(static_cast<std::size_t>(std::max<int64_t>(cm, 1)));
        if (cm > 0) {
            k_prune_scatter<<<blocks_for(cm, kT), kT, 0, s>>>(cm, F.c_col.get(), F.cv.get(), flags, slot,
                                                             F.keep_pos.get(), C.co.get(), C.va.get());
            check_launch(ctx_);
        }
        k_pruned_offsets<<<blocks_for(nc + 1, kT), kT, 0, s>>>(nc, F.c_off.get(), slot, C.ro.get());
        check_launch(ctx_);
    }
    if (read_status(ctx_) & kRefreshInvalid) return false;   // synchronises
    phase("pruning");
    // the coarse operator back to the host for the next level's C/F splitting
    // (the offsets and columns are non-negative, so their int bits are the
    // uint32 values)
    coarse.n = coarse_n;
    coarse.ro.resize(static_cast<std::size_t>(nc) + 1);
    coarse.co.resize(static_cast<std::size_t>(C.nnz));
    coarse.va.resize(static_cast<std::size_t>(C.nnz));
    download(C.ro.get(), coarse.ro.data(), sizeof(int) * (static_cast<std::size_t>(nc) + 1));
    download(C.co.get(), coarse.co.data(), sizeof(int) * static_cast<std::size_t>(C.nnz));
    download(C.va.get(), coarse.va.data(), sizeof(double) * static_cast<std::size_t>(C.nnz));
    C.inv_diag.resize(static_cast<std::size_t>(nc));
    phase("download");
    return true;
}

std::unique_ptr<DevRefresh> DeviceGalerkin::take(int levels) {
    if (static_cast<int>(R_->L.size()) < levels) return nullptr;
    R_->L.resize(static_cast<std::size_t>(levels));
    R_->bounds.resize(static_cast<std::size_t>(levels));
    return std::move(R_);
}

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
    // per-phase times with CFDXG_SETUP_PROFILE (synchronising)
    static const bool profile = std::getenv("CFDXG_SETUP_PROFILE") != nullptr;
    double tp = wall_seconds();
    auto phase = [&](const char* what) {
        if (!profile) return;
        CFDXG_CUDA(cudaStreamSynchronize(s));
        const double t = wall_seconds();
        std::fprintf(stderr, "[cfdxg refresh] %s %.4fs\n", what, t - tp);
        tp = t;
    };
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
                const int splits = choose_splits(F.n, static_cast<int64_t>(F.ap.size()));
                k_ap_rows<<<galerkin_grid(F.n, splits), 32 * kWarpRows, 0, s>>>(
                    F.n, F.ro.get(), F.co.get(), F.va.get(), F.p_off.get(), F.p_col.get(), F.p_val.get(),
                    F.ap_off.get(), F.ap_col.get(), F.ap.get(), splits, st);
                check_launch(ctx);
            }
            {
                ProfScope ps(ctx, "refresh_galerkin_c", 0.0);
                const int splits = choose_splits(F.n_coarse, static_cast<int64_t>(F.cv.size()));
                k_c_rows<<<galerkin_grid(F.n_coarse, splits), 32 * kWarpRows, 0, s>>>(
                    F.n_coarse, F.t_off.get(), F.t_row.get(), F.t_pos.get(), F.p_off.get(), F.p_val.get(),
                    F.ap_off.get(), F.ap_col.get(), F.ap.get(), F.c_off.get(), F.c_col.get(), F.cv.get(), splits, st);
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
    phase("Galerkin products and diagonals");
    R.bounds.zero(s);
    {
        ProfScope ps_bounds(ctx, "refresh_gershgorin", 0.0);
        int64_t most = 0;
        for (std::size_t l = 0; l < nl; ++l) most = std::max<int64_t>(most, R.L[l].n);
        if (static_cast<int64_t>(R.sqrt_diag.size()) < most) R.sqrt_diag.resize(static_cast<std::size_t>(most));
        for (std::size_t l = 0; l < nl; ++l) {
            DevRefreshLevel& L = R.L[l];
            k_sqrt_diagonal<<<blocks_for(L.n, kT), kT, 0, s>>>(L.n, L.inv_diag.get(), R.sqrt_diag.get(),
                                                               R.bounds.get() + l);
            if (L.nnz >= 32 * static_cast<int64_t>(L.n))
                k_gershgorin_warp<<<std::max(1, std::min(blocks_for(L.n, 8), 148 * 32)), 256, 0, s>>>(
                    L.n, L.ro.get(), L.co.get(), L.va.get(), R.sqrt_diag.get(), R.bounds.get() + l);
            else
                k_gershgorin<<<blocks_for(L.n, kT), kT, 0, s>>>(L.n, L.ro.get(), L.co.get(), L.va.get(),
                                                                R.sqrt_diag.get(), R.bounds.get() + l);
            check_launch(ctx);
        }
    }
    std::vector<double> bounds(nl);
    R.bounds.download(bounds.data(), s);
    const int status = read_status(ctx);   // synchronises the stream
    phase("damping bounds");
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
    phase("commit");
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
