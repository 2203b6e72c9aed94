// vcycle.cu -- device AMG hierarchy and the V-cycle (damped-Jacobi V(pre,post)).
//
// The FP64 instantiation follows MatrixFreeVcyclePreconditioner::vcycle /
// smooth / smooth_coarsest (core/linalg/amg_preconditioner.h:2369-2443,
// 2564-2666) operation by operation: every row sum runs in CSR order from 0.0,
// the restriction gathers P^T rows in increasing fine-row order (the order in
// which the reference's scatter adds them), the prolongation adds P entries to
// x one at a time, and the first sweep from x = 0 skips the product A*0 = 0.
// It therefore returns the reference's z = M^-1 r bit for bit.  The FP32
// instantiation runs the same cycle in single precision with FP32
// accumulation and replaces the bottom of the hierarchy by an FP64 dense
// solve at the first level with <= coarse_dense_limit rows.
//
// Level 0 is launched directly with the caller's vectors; levels >= 1 are
// captured once into a CUDA graph with fixed buffers and replayed.
//
// Under the constant null space (constant_null_space) the cycle removes the
// mean from its input and output, after every sweep, after the restriction
// and after the prolongation, and the <= 16-row coarsest level solves the
// system bordered by a row and a column of ones (amg_preconditioner.h:1197-1201,
// 2382, 2406, 2430, 2440, 2590-2664); the FP32 cycle's dense coarse inverse
// is then the leading block of the bordered matrix's inverse.
#include <cub/device/device_scan.cuh>
#include <cusolverDn.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <limits>
#include <type_traits>

#include "nullspace.cuh"
#include "objects.h"

namespace cfdxg {

namespace {

constexpr int kT = 256;
constexpr int kCoarseSweeps = 24;   // amg_preconditioner.h:2585
constexpr int kFp32CoarsePre = 0;   // FP32 cycle on levels >= 1: V(0,1)
constexpr int kFp32CoarsePost = 1;
constexpr int kDenseDirectLimit = 16;

template <class T>
__device__ __forceinline__ bool finite_(T v) { return isfinite(v); }

// First sweep from x = 0 (A*0 = 0): x = 0 + omega * (inv_diag * (r - 0)).
template <class T, class R>
__global__ void k_sweep_zero(int n, T omega, const T* __restrict__ inv_diag, const R* __restrict__ r,
                             T* __restrict__ r_copy, T* __restrict__ x, int* status) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const T ri = static_cast<T>(r[i]);
    if (r_copy) r_copy[i] = ri;
    const T delta = inv_diag[i] * (ri - T(0));
    const T xi = T(0) + omega * delta;
    x[i] = xi;
    if (!finite_(xi)) atomicOr(status, kStatusNonFinite);
}

// Row reductions.  TPR threads cooperate on one row; TPR == 1 sums the row
// sequentially in CSR order (the reference's order).  TPR > 1 gives each
// thread the entries k = lane, lane + TPR, ... and combines the partial sums
// with a fixed xor butterfly, so results are deterministic run to run.
// Measured alternatives that were slower on the 64^3 tet hierarchy: 16-byte
// chunks of four entries per lane (~5%), eight lanes per short row with the
// sum formed in order through shuffles (~4x), and a sliced-ELL copy of the
// fine level (32-row slices, column-major; ~10%).
//
// CI is the column index type: int (absolute columns, base 0) or int16_t
// (offsets from the row, base = the row index).
// A stored value as T: FP32 / FP64 as is, FP16 (half_values) widened.
template <class T, class VS>
__device__ __forceinline__ T ldv(const VS* __restrict__ p, int k) {
    if constexpr (std::is_same<VS, __half>::value) return static_cast<T>(__half2float(p[k]));
    else return p[k];
}

// NWARPS: warps of the launching block (rows wider than a warp are combined
// through a per-warp shared array of that size).
template <class T, int TPR, int NWARPS>
__device__ __forceinline__ T row_reduce_n(T s, int lane) {
    if (TPR > 1) {
        constexpr int W = TPR < 32 ? TPR : 32;
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, W);
    }
    if constexpr (TPR > 32) {
        // rows spread over TPR / 32 warps of the block (levels with few, long
        // rows): warp partials summed in warp order by the row's first thread
        __shared__ T part[NWARPS];
        const int warp = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) part[warp] = s;
        __syncthreads();
        if (lane == 0) {
            T t = part[warp];
#pragma unroll
            for (int q = 1; q < TPR / 32; ++q) t += part[warp + q];
            s = t;
        }
    }
    return s;
}

template <class T, int TPR>
__device__ __forceinline__ T row_reduce(T s, int lane) { return row_reduce_n<T, TPR, kT / 32>(s, lane); }

template <class T, int TPR, class CI = int, class VS = T>
__device__ __forceinline__ T row_dot(int b, int e, int lane, const CI* __restrict__ co,
                                     const VS* __restrict__ va, const T* __restrict__ x, int base = 0) {
    T s = T(0);
    // unrolled so several independent (value, column, x) loads are in flight;
    // the additions stay in the same sequential order
#pragma unroll 4
    for (int k = b + lane; k < e; k += TPR) s += ldv<T>(va, k) * __ldg(x + (base + static_cast<int>(co[k])));
    return row_reduce<T, TPR>(s, lane);
}

// The first PF entries a lane visits (k = b + lane + q TPR), loaded before the
// kernel waits for its predecessor on the stream: within a cycle the
// predecessor of a sweep or residual is always another cycle kernel, which
// writes vectors only, never the level's matrix.  row_dot_head then sums
// them, and the rest of the lane's entries, in row_dot's order.
template <class T, class CI, int PF>
struct RowHead {
    T v[PF];
    CI c[PF];
};

template <class T, int TPR, class CI, int PF, class VS = T>
__device__ __forceinline__ void row_head_load(RowHead<T, CI, PF>& h, int b, int e, int lane,
                                              const CI* __restrict__ co, const VS* __restrict__ va) {
#pragma unroll
    for (int q = 0; q < PF; ++q) {
        const int k = b + lane + q * TPR;
        h.v[q] = k < e ? ldv<T>(va, k) : T(0);
        h.c[q] = k < e ? co[k] : CI(0);
    }
}

template <class T, int TPR, class CI, int PF, class VS = T>
__device__ __forceinline__ T row_dot_head(const RowHead<T, CI, PF>& h, int b, int e, int lane,
                                          const CI* __restrict__ co, const VS* __restrict__ va,
                                          const T* __restrict__ x, int base) {
    T s = T(0);
#pragma unroll
    for (int q = 0; q < PF; ++q)
        if (b + lane + q * TPR < e) s += h.v[q] * __ldg(x + (base + static_cast<int>(h.c[q])));
    int k = b + lane + PF * TPR;
    if constexpr (TPR > 1) {
        // Shared rows are long: take the lane's entries eight at a time --
        // all eight columns and values, then all eight x gathers, then the
        // products in entry order (the same additions as the loop below) --
        // so eight gathers are in flight per lane instead of four (the
        // coarse sweeps stall on load latency, not on bandwidth).
        constexpr int B = 8;
        for (; k + (B - 1) * TPR < e; k += B * TPR) {
            CI c[B];
            T v[B], xv[B];
#pragma unroll
            for (int q = 0; q < B; ++q) {
                c[q] = co[k + q * TPR];
                v[q] = ldv<T>(va, k + q * TPR);
            }
#pragma unroll
            for (int q = 0; q < B; ++q) xv[q] = __ldg(x + (base + static_cast<int>(c[q])));
#pragma unroll
            for (int q = 0; q < B; ++q) s += v[q] * xv[q];
        }
    }
#pragma unroll 4
    for (; k < e; k += TPR)
        s += ldv<T>(va, k) * __ldg(x + (base + static_cast<int>(co[k])));
    return row_reduce<T, TPR>(s, lane);
}

// Shared rows prefetch four entries per lane.  On one-thread rows (the fine
// level) the prefetch measured 5% slower (18.7 vs 17.7 us per FP32 sweep):
// there the kernel waits first and issues its own row loads early instead.
template <int TPR>
__host__ __device__ constexpr int head_entries() { return TPR == 1 ? 1 : 4; }

template <class CI>
__device__ __forceinline__ int column_base(int row) { return sizeof(CI) == 2 ? row : 0; }

// x_out = x + omega * (inv_diag * (r - A x)).  With FP16 values (VS = __half)
// the row sum is formed on the stored fractions and scaled once by rscale.
template <class T, class XO, int TPR, class CI, class VS>
__global__ void k_sweep(int n, const int* __restrict__ ro, const CI* __restrict__ co,
                        const VS* __restrict__ va, const T* __restrict__ rscale, const T* __restrict__ inv_diag,
                        const T* __restrict__ r, const T* __restrict__ x, XO* __restrict__ xo,
                        T omega, int* status) {
    pdl_trigger();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = g / TPR, lane = g % TPR;
    const bool valid = i < n;
    // One thread per row: the row's own r, x and inverse diagonal are loaded
    // before the row walk so their latency overlaps it (17.5 vs 19.4 us per
    // fine-level FP32 sweep at 64^3); with shared rows the extra registers
    // cost more than they hide.
    T ri = T(0), xi = T(0), di = T(0);
    T s;
    if constexpr (TPR == 1) {
        pdl_wait();
        if (valid) { ri = r[i]; xi = x[i]; di = inv_diag[i]; }
        s = row_dot<T, TPR, CI, VS>(valid ? ro[i] : 0, valid ? ro[i + 1] : 0, lane, co, va, x, column_base<CI>(i));
    } else {
        const int b = valid ? ro[i] : 0, e = valid ? ro[i + 1] : 0;
        RowHead<T, CI, head_entries<TPR>()> head;
        row_head_load<T, TPR, CI, head_entries<TPR>(), VS>(head, b, e, lane, co, va);
        pdl_wait();
        s = row_dot_head<T, TPR, CI, head_entries<TPR>(), VS>(head, b, e, lane, co, va, x, column_base<CI>(i));
    }
    if (!valid || lane != 0) return;
    if constexpr (TPR > 1) { ri = r[i]; xi = x[i]; di = inv_diag[i]; }
    if constexpr (std::is_same<VS, __half>::value) s = s * rscale[i];
    const T delta = di * (ri - s);
    const T xn = xi + omega * delta;
    xo[i] = static_cast<XO>(xn);
    if (!finite_(xn)) atomicOr(status, kStatusNonFinite);
}

template <class T, int TPR, class CI, class VS>
__global__ void k_residual(int n, const int* __restrict__ ro, const CI* __restrict__ co,
                           const VS* __restrict__ va, const T* __restrict__ rscale, const T* __restrict__ r,
                           const T* __restrict__ x, T* __restrict__ res) {
    pdl_trigger();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = g / TPR, lane = g % TPR;
    const bool valid = i < n;
    T ri = T(0);
    T s;
    if constexpr (TPR == 1) {
        pdl_wait();
        if (valid) ri = r[i];
        s = row_dot<T, TPR, CI, VS>(valid ? ro[i] : 0, valid ? ro[i + 1] : 0, lane, co, va, x, column_base<CI>(i));
    } else {
        const int b = valid ? ro[i] : 0, e = valid ? ro[i + 1] : 0;
        RowHead<T, CI, head_entries<TPR>()> head;
        row_head_load<T, TPR, CI, head_entries<TPR>(), VS>(head, b, e, lane, co, va);
        pdl_wait();
        s = row_dot_head<T, TPR, CI, head_entries<TPR>(), VS>(head, b, e, lane, co, va, x, column_base<CI>(i));
    }
    if (!valid || lane != 0) return;
    if constexpr (TPR > 1) ri = r[i];
    if constexpr (std::is_same<VS, __half>::value) s = s * rscale[i];
    res[i] = ri - s;
}

// coarse_r = P^T res, rows of P^T in increasing fine-row order
template <class T, int TPR>
__global__ void k_restrict(int nc, const int* __restrict__ r_off, const int* __restrict__ r_row,
                           const T* __restrict__ r_val, const T* __restrict__ res, T* __restrict__ rc) {
    // P^T is fixed for the hierarchy's lifetime: its entries are loaded
    // before waiting for the kernel that produced res
    pdl_trigger();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = g / TPR, lane = g % TPR;
    const bool valid = c < nc;
    const int b = valid ? r_off[c] : 0, e = valid ? r_off[c + 1] : 0;
    RowHead<T, int, 4> head;
    row_head_load<T, TPR, int, 4>(head, b, e, lane, r_row, r_val);
    pdl_wait();
    const T s = row_dot_head<T, TPR, int, 4>(head, b, e, lane, r_row, r_val, res, 0);
    if (valid && lane == 0) rc[c] = s;
}

// x += P xc.  TPR == 1 adds the entries to x one by one in P's row order (the
// reference's order); TPR > 1 forms the row sum cooperatively (deterministic
// butterfly, as row_dot) and adds it once.
// With ASSIGN the level's x is taken as zero (no pre-sweeps: the cycle would
// otherwise clear it first) and x = 0 + P xc is written without reading x --
// the same arithmetic as clearing x and adding, one graph node fewer per level.
template <class T, int TPR, bool ASSIGN = false>
__global__ void k_prolong(int n, const int* __restrict__ p_off, const int* __restrict__ p_col,
                          const T* __restrict__ p_val, const T* __restrict__ xc, T* __restrict__ x,
                          int* status) {
    // P is fixed for the hierarchy's lifetime: its entries are loaded before
    // waiting for the kernels that produced x and xc
    pdl_trigger();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = g / TPR, lane = g % TPR;
    const bool valid = i < n;
    const int b = valid ? p_off[i] : 0, e = valid ? p_off[i + 1] : 0;
    RowHead<T, int, 4> head;
    row_head_load<T, TPR, int, 4>(head, b, e, lane, p_col, p_val);
    pdl_wait();
    if constexpr (TPR == 1) {
        if (!valid) return;
        T v = ASSIGN ? T(0) : x[i];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (b + q < e) v += head.v[q] * __ldg(xc + head.c[q]);
        for (int q = b + 4; q < e; ++q) v += p_val[q] * __ldg(xc + p_col[q]);
        x[i] = v;
        if (!finite_(v)) atomicOr(status, kStatusNonFinite);
    } else {
        const T s = row_dot_head<T, TPR, int, 4>(head, b, e, lane, p_col, p_val, xc, 0);
        if (!valid || lane != 0) return;
        const T v = (ASSIGN ? T(0) : x[i]) + s;
        x[i] = v;
        if (!finite_(v)) atomicOr(status, kStatusNonFinite);
    }
}

template <class T, class XO>
__global__ void k_copy_cast(int n, const T* __restrict__ a, XO* __restrict__ b) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = static_cast<XO>(a[i]);
}

// Reference dense pivoted solve of the coarsest level (amg_preconditioner.h:2592-2663),
// executed by one thread in the reference's order; under the constant null
// space (ns = 1) the system is bordered by a row and a column of ones and the
// mean of the solution is removed, summed in order.
template <class T>
__global__ void k_dense_lu_reference(int n, const int* __restrict__ ro, const int* __restrict__ co,
                                     const T* __restrict__ va, const T* __restrict__ r,
                                     T* __restrict__ x, int ns, int* status) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    constexpr int kMax = kDenseDirectLimit + 1;
    double m[kMax * kMax];
    double b[kMax];
    double sol[kMax];
    const int sn = n + (ns ? 1 : 0);
    for (int q = 0; q < sn * sn; ++q) m[q] = 0.0;
    for (int i = 0; i < sn; ++i) b[i] = 0.0;
    for (int i = 0; i < n; ++i) {
        b[i] = static_cast<double>(r[i]);
        for (int k = ro[i]; k < ro[i + 1]; ++k) m[i * sn + co[k]] += static_cast<double>(va[k]);
    }
    if (ns)
        for (int i = 0; i < n; ++i) {
            m[i * sn + n] = 1.0;
            m[n * sn + i] = 1.0;
        }
    double matrix_scale = 0.0;
    for (int q = 0; q < sn * sn; ++q) {
        const double a = fabs(m[q]);
        matrix_scale = (matrix_scale < a) ? a : matrix_scale;
    }
    const double pivot_tol = 128.0 * 2.220446049250313080847e-16 * (1.0 < matrix_scale ? matrix_scale : 1.0);
    for (int k = 0; k < sn; ++k) {
        int pivot = k;
        double pivot_abs = fabs(m[k * sn + k]);
        for (int i = k + 1; i < sn; ++i) {
            const double c = fabs(m[i * sn + k]);
            if (c > pivot_abs) { pivot_abs = c; pivot = i; }
        }
        if (!isfinite(pivot_abs) || pivot_abs <= pivot_tol) { atomicOr(status, kStatusNonFinite); return; }
        if (pivot != k) {
            for (int j = k; j < sn; ++j) { const double t = m[k * sn + j]; m[k * sn + j] = m[pivot * sn + j]; m[pivot * sn + j] = t; }
            const double t = b[k]; b[k] = b[pivot]; b[pivot] = t;
        }
        const double diagonal = m[k * sn + k];
        for (int i = k + 1; i < sn; ++i) {
            const double factor = m[i * sn + k] / diagonal;
            if (!isfinite(factor)) { atomicOr(status, kStatusNonFinite); return; }
            m[i * sn + k] = 0.0;
            for (int j = k + 1; j < sn; ++j) m[i * sn + j] -= factor * m[k * sn + j];
            b[i] -= factor * b[k];
        }
    }
    for (int ii = sn - 1; ii >= 0; --ii) {
        double sum = b[ii];
        for (int j = ii + 1; j < sn; ++j) sum -= m[ii * sn + j] * sol[j];
        const double diagonal = m[ii * sn + ii];
        if (!isfinite(diagonal) || fabs(diagonal) <= pivot_tol) { atomicOr(status, kStatusNonFinite); return; }
        sol[ii] = sum / diagonal;
        if (!isfinite(sol[ii])) { atomicOr(status, kStatusNonFinite); return; }
    }
    if (ns) {
        double mean = 0.0;
        for (int i = 0; i < n; ++i) mean += sol[i];
        mean /= static_cast<double>(n);
        for (int i = 0; i < n; ++i) sol[i] -= mean;
    }
    for (int i = 0; i < n; ++i) x[i] = static_cast<T>(sol[i]);
}

// x = Ainv * r, one warp per row: the inverse (formed in FP64) is read as
// FP32 -- half the bytes of the largest single read of the FP32 cycle -- and
// the products are summed in FP64.
template <class T, class S>
__global__ void k_dense_inverse_apply(int n, const S* __restrict__ inv, const T* __restrict__ r,
                                      T* __restrict__ x, int* status) {
    pdl_entry();
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    double s = 0.0;
    const S* row = inv + static_cast<size_t>(warp) * n;
#pragma unroll 4
    for (int j = lane; j < n; j += 32) s += static_cast<double>(row[j]) * static_cast<double>(r[j]);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) {
        x[warp] = static_cast<T>(s);
        if (!isfinite(s)) atomicOr(status, kStatusNonFinite);
    }
}

// ---- dense coarse inverse (LU with partial pivoting, cuSOLVER) ----
// A^T, dense column-major with leading dimension ld (so element (j, i) of the
// array is a_ij): the LU path solves A^T X = I, whose column-major X read
// row-major is A^-1.  With ld = n + 1 and `border`, the matrix is bordered by
// a row and a column of ones (a zero in the corner).
__global__ void k_dense_init_t(int n, int ld, const int* ro, const int* co, const double* va, int border,
                               double* at) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = ro[i]; k < ro[i + 1]; ++k) at[static_cast<size_t>(i) * ld + co[k]] += va[k];
    if (border) {
        at[static_cast<size_t>(i) * ld + n] = 1.0;
        at[static_cast<size_t>(n) * ld + i] = 1.0;
    }
}

__global__ void k_identity(int64_t n, double* x) {
    const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx < n * n) x[idx] = (idx / n == idx % n) ? 1.0 : 0.0;
}

// b (n x n) = the leading n x n block of a (row-major, leading dimension ld)
template <class S>
__global__ void k_dense_block_copy(int n, int ld, const double* __restrict__ a, S* __restrict__ b) {
    const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= static_cast<int64_t>(n) * n) return;
    const int64_t i = idx / n, j = idx % n;
    b[idx] = static_cast<S>(a[i * ld + j]);
}

// flag = 1 when the N x N matrix a is not symmetric: |a_ij - a_ji| above
// 1e-12 of the pair's magnitude plus 1e-14 of sqrt(|a_ii a_jj|) (the coarse
// Galerkin operators of a symmetric system differ from symmetry only by the
// rounding of their sums, which leaves entries cancelled to near zero with
// differences far above their own size but far below the diagonal's)
__global__ void k_symmetry_check(int N, const double* __restrict__ a, int* flag) {
    const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= static_cast<int64_t>(N) * N) return;
    const int64_t i = idx / N, j = idx % N;
    if (j <= i) return;
    const double x = a[i * N + j], y = a[j * N + i];
    const double scale = sqrt(fabs(a[i * N + i]) * fabs(a[j * N + j]));
    if (!(fabs(x - y) <= 1e-12 * (fabs(x) + fabs(y)) + 1e-14 * scale)) atomicOr(flag, 1);
}

// b (n x n, row-major) = the symmetric matrix whose lower triangle is held
// column-major in a (leading dimension ld)
template <class S>
__global__ void k_dense_sym_copy(int n, int ld, const double* __restrict__ a, S* __restrict__ b) {
    const int64_t idx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= static_cast<int64_t>(n) * n) return;
    const int64_t i = idx / n, j = idx % n;
    const int64_t lo = i < j ? i : j, hi = i < j ? j : i;
    b[idx] = static_cast<S>(a[lo * ld + hi]);
}

#define CFDXG_TPR_SWITCH(tpr, ...)                            \
    switch (tpr) {                                               \
        case 1: { constexpr int TPR = 1; __VA_ARGS__; } break;   \
        case 2: { constexpr int TPR = 2; __VA_ARGS__; } break;   \
        case 4: { constexpr int TPR = 4; __VA_ARGS__; } break;   \
        case 8: { constexpr int TPR = 8; __VA_ARGS__; } break;   \
        case 16: { constexpr int TPR = 16; __VA_ARGS__; } break; \
        case 32: { constexpr int TPR = 32; __VA_ARGS__; } break; \
        case 64: { constexpr int TPR = 64; __VA_ARGS__; } break; \
        case 128: { constexpr int TPR = 128; __VA_ARGS__; } break; \
        default: { constexpr int TPR = 256; __VA_ARGS__; } break; \
    }

// Algorithmic (compulsory) bytes of one launch; accumulated into the graph
// total while a capture is in progress.
thread_local double* t_capture_bytes = nullptr;

inline double account(double bytes) {
    if (t_capture_bytes) *t_capture_bytes += bytes;
    return bytes;
}

template <class T>
const char* tname(const char* fp64, const char* fp32) { return sizeof(T) == 8 ? fp64 : fp32; }

// Bytes of one stored nonzero of A (value + column) and per row (offset, and
// the row scale of FP16 values).
template <class T>
double nonzero_bytes(const DevLevel<T>& L) { return (L.half ? 2.0 : sizeof(T)) + (L.narrow ? 2.0 : 4.0); }
template <class T>
double row_bytes(const DevLevel<T>& L) { return 4.0 + (L.half ? sizeof(T) : 0.0); }

// Calls go(columns, values, row_scale) with the level's storage types.
template <class T, class Go>
void with_level_storage(const DevLevel<T>& L, Go&& go) {
    if constexpr (std::is_same<T, float>::value) {
        if (L.half) {
            if (L.narrow) go(L.co16.get(), L.vh.get(), L.rscale.get());
            else go(L.co.get(), L.vh.get(), L.rscale.get());
            return;
        }
    }
    if (L.narrow) go(L.co16.get(), L.va.get(), static_cast<const T*>(nullptr));
    else go(L.co.get(), L.va.get(), static_cast<const T*>(nullptr));
}

template <class T, class XO>
void launch_sweep(cfdxg_context* ctx, const DevLevel<T>& L, const T* r, const T* x, XO* xo, T omega, int* status) {
    // A values + columns, row offsets (+ scales), x / r / inv_diag reads, x_out write
    const double bytes = account(nonzero_bytes(L) * L.nnz + row_bytes(L) * L.n + 4.0 + 3.0 * sizeof(T) * L.n +
                                 sizeof(XO) * L.n);
    ProfScope ps(ctx, tname<T>("jacobi_sweep_fp64_L0", "jacobi_sweep_fp32_L0"), bytes);
    const int grid = blocks_for(static_cast<int64_t>(L.n) * L.tpr, kT);
    with_level_storage(L, [&](const auto* co, const auto* va, const T* rs) {
        using CI = std::remove_cv_t<std::remove_pointer_t<decltype(co)>>;
        using VS = std::remove_cv_t<std::remove_pointer_t<decltype(va)>>;
        CFDXG_TPR_SWITCH(L.tpr, (launch_pdl(ctx->stream, k_sweep<T, XO, TPR, CI, VS>, grid, kT, L.n, L.ro.get(), co,
                                            va, rs, L.inv_diag.get(), r, x, xo, omega, status)));
    });
    check_launch(ctx);
}

template <class T>
void launch_residual(cfdxg_context* ctx, const DevLevel<T>& L, const T* r, const T* x, T* res) {
    const double bytes = account(nonzero_bytes(L) * L.nnz + row_bytes(L) * L.n + 4.0 + 3.0 * sizeof(T) * L.n);
    ProfScope ps(ctx, tname<T>("residual_fp64_L0", "residual_fp32_L0"), bytes);
    const int grid = blocks_for(static_cast<int64_t>(L.n) * L.tpr, kT);
    with_level_storage(L, [&](const auto* co, const auto* va, const T* rs) {
        using CI = std::remove_cv_t<std::remove_pointer_t<decltype(co)>>;
        using VS = std::remove_cv_t<std::remove_pointer_t<decltype(va)>>;
        CFDXG_TPR_SWITCH(L.tpr, (launch_pdl(ctx->stream, k_residual<T, TPR, CI, VS>, grid, kT, L.n, L.ro.get(), co,
                                            va, rs, r, x, res)));
    });
    check_launch(ctx);
}

template <class T>
void launch_restrict(cfdxg_context* ctx, const DevLevel<T>& L, const T* res, T* rc) {
    const double pnnz = static_cast<double>(L.r_row.size());
    const double bytes = account((sizeof(T) + 4.0) * pnnz + 4.0 * (L.nc + 1) + sizeof(T) * (L.n + L.nc));
    ProfScope ps(ctx, tname<T>("restrict_fp64_L0", "restrict_fp32_L0"), bytes);
    const int64_t threads = static_cast<int64_t>(L.nc) * L.tpr_r;
    CFDXG_TPR_SWITCH(L.tpr_r, (launch_pdl(ctx->stream, k_restrict<T, TPR>, blocks_for(threads, kT), kT, 
        L.nc, L.r_off.get(), L.r_row.get(), L.r_val.get(), res, rc)));
    check_launch(ctx);
}

template <class T>
void launch_prolong(cfdxg_context* ctx, const DevLevel<T>& L, const T* xc, T* x, int* status,
                    bool assign = false) {
    const double pnnz = static_cast<double>(L.p_col.size());
    const double bytes = account((sizeof(T) + 4.0) * pnnz + 4.0 * (L.n + 1) +
                                 sizeof(T) * (L.nc + (assign ? 1.0 : 2.0) * L.n));
    ProfScope ps(ctx, tname<T>("prolong_fp64_L0", "prolong_fp32_L0"), bytes);
    const int64_t threads = static_cast<int64_t>(L.n) * L.tpr_p;
    if (assign) {
        CFDXG_TPR_SWITCH(L.tpr_p, (launch_pdl(ctx->stream, k_prolong<T, TPR, true>, blocks_for(threads, kT), kT,
                                              L.n, L.p_off.get(), L.p_col.get(), L.p_val.get(), xc, x, status)));
    } else {
        CFDXG_TPR_SWITCH(L.tpr_p, (launch_pdl(ctx->stream, k_prolong<T, TPR, false>, blocks_for(threads, kT), kT,
                                              L.n, L.p_off.get(), L.p_col.get(), L.p_val.get(), xc, x, status)));
    }
    check_launch(ctx);
}

// Threads per row of A: the largest power of two with at least eight entries
// per thread, up to a warp; past a warp (up to four warps) only while the
// level has too few rows to fill two waves of the GPU (148 SMs x 2048
// threads).  Measured per level on the 64^3 tet hierarchy (FP32 and FP64,
// every power of two from 1 to 256): this picks the fastest split or one
// within 3% of it on every level; 256 threads per row was never the fastest.
int choose_tpr(int64_t nnz, int64_t rows, bool reference_order) {
    if (reference_order || rows == 0) return 1;
    const double avg = static_cast<double>(nnz) / static_cast<double>(rows);
    int tpr = 1;
    while (tpr < 32 && avg >= 16.0 * tpr) tpr *= 2;
    while (tpr >= 32 && tpr < 128 && static_cast<double>(rows) * tpr < 2.0 * 148.0 * 2048.0 && avg >= 8.0 * tpr)
        tpr *= 2;
    return tpr;
}

// Threads per row of a sparsified smoothing operator (rows of 9-70 entries
// at 64^3): the largest power of two up to a warp with at least
// kSparseRowEntries entries per thread.  Eight measured 6.68 ms per 64^3 FP32
// solve against 6.89 for sixteen (the rule of the Galerkin levels) and 6.80
// for four; 18.9 against 19.2 and 19.4 ms on the 4.2 M-cell boundary layer.
constexpr int kSparseRowEntries = 8;
int choose_sparse_tpr(int64_t nnz, int64_t rows) {
    if (rows == 0) return 1;
    const double avg = static_cast<double>(nnz) / static_cast<double>(rows);
    int tpr = 1;
    while (tpr < 32 && avg >= static_cast<double>(kSparseRowEntries) * tpr) tpr *= 2;
    return tpr;
}

// Transfer operators (rows of P or P^T): as choose_tpr, then more threads per
// row while the level has too few rows to fill the GPU (ragged rows on the deep
// levels otherwise leave a few threads walking long rows alone).
int choose_transfer_tpr(int64_t nnz, int64_t rows, bool reference_order) {
    int tpr = choose_tpr(nnz, rows, reference_order);
    if (reference_order) return tpr;
    tpr = std::min(tpr, 32);
    while (tpr < 32 && static_cast<double>(rows) * tpr < 148.0 * 1024.0) tpr *= 2;
    return tpr;
}

template <class T>
void upload_level_values(cfdxg_context* ctx, DevLevel<T>& D, const AmgLevel& H) {
    if (D.half) {
        // FP16 fractions of each row's largest magnitude (the same rounding as k_quantize_rows)
        const int n = static_cast<int>(H.A.n);
        std::vector<__half> q(H.A.va.size());
        std::vector<T> sc(n);
        for (int i = 0; i < n; ++i) {
            double m = 0.0;
            for (uint32_t k = H.A.ro[i]; k < H.A.ro[i + 1]; ++k) m = std::max(m, std::fabs(H.A.va[k]));
            const float s = m > 0.0 ? static_cast<float>(m) : 1.0f;
            sc[i] = static_cast<T>(s);
            for (uint32_t k = H.A.ro[i]; k < H.A.ro[i + 1]; ++k)
                q[k] = __float2half_rn(static_cast<float>(H.A.va[k] / static_cast<double>(s)));
        }
        D.vh.upload(q, ctx->stream);
        D.rscale.upload(sc, ctx->stream);
        D.va.release();
    } else {
        std::vector<T> tmp(H.A.va.size());
        for (std::size_t k = 0; k < tmp.size(); ++k) tmp[k] = static_cast<T>(H.A.va[k]);
        D.va.upload(tmp, ctx->stream);
    }

    std::vector<T> d(H.inv_diag.size());
    for (std::size_t k = 0; k < d.size(); ++k) d[k] = static_cast<T>(H.inv_diag[k]);
    D.inv_diag.upload(d, ctx->stream);
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
}

// Narrow columns (int16 offsets from the row) for a level whose every
// |column - row| fits; the coarsest level keeps absolute columns for its
// direct solvers.
template <class T>
void upload_columns(cfdxg_context* ctx, DevLevel<T>& D, const AmgLevel& H, bool allow_narrow) {
    const int n = static_cast<int>(H.A.n);
    bool narrow = allow_narrow;
    for (int i = 0; i < n && narrow; ++i)
        for (uint32_t k = H.A.ro[i]; k < H.A.ro[i + 1]; ++k) {
            const int64_t d = static_cast<int64_t>(H.A.co[k]) - i;
            if (d < INT16_MIN || d > INT16_MAX) { narrow = false; break; }
        }
    D.narrow = narrow;
    if (narrow) {
        std::vector<int16_t> c16(H.A.co.size());
        for (int i = 0; i < n; ++i)
            for (uint32_t k = H.A.ro[i]; k < H.A.ro[i + 1]; ++k)
                c16[k] = static_cast<int16_t>(static_cast<int64_t>(H.A.co[k]) - i);
        D.co16.upload(c16, ctx->stream);
        D.co.release();
    } else {
        std::vector<int> co(H.A.co.begin(), H.A.co.end());
        D.co.upload(co, ctx->stream);
        D.co16.release();
    }
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
}

template <class T>
void upload_level(cfdxg_context* ctx, DevLevel<T>& D, const AmgLevel& H, bool with_transfer,
                  const UploadOptions& opt) {
    const bool reference_order = opt.reference_order;
    cudaStream_t s = ctx->stream;
    D.n = static_cast<int>(H.A.n);
    D.nnz = static_cast<int>(H.A.co.size());
    D.tpr = choose_tpr(D.nnz, D.n, reference_order);
    std::vector<int> ro(H.A.ro.begin(), H.A.ro.end());
    D.ro.upload(ro, s);
    // Narrow columns pay on short rows (one thread per row: 21.1 vs 22.5 us per
    // fine-level FP32 sweep at 64^3); on the long rows that a warp shares they
    // measured 10-20% slower (58.9 -> 70.6 us on the 77,039-row level), so
    // those keep int32 columns.
    upload_columns(ctx, D, H, with_transfer && opt.narrow_columns && D.tpr == 1);
    // FP16 values on the shared-row levels (the dense coarse operators: 475 vs
    // 501 us per FP32 cycle of levels >= 1 at 64^3, iterations unchanged); on
    // one-thread rows the conversion cost more than the bytes saved
    // (18.1 vs 17.7 us per fine-level sweep)
    D.half = std::is_same<T, float>::value && opt.half_values && with_transfer && D.tpr > 1;
    upload_level_values(ctx, D, H);
    D.r.resize(D.n); D.x.resize(D.n); D.x2.resize(D.n); D.res.resize(D.n);
    if (with_transfer) {
        const int n = D.n;
        int nc = 0;
        for (const uint32_t c : H.p_col) nc = std::max<int>(nc, static_cast<int>(c) + 1);
        nc = std::max<int>(nc, static_cast<int>(H.plan.n_coarse));
        D.nc = nc;
        D.tpr_r = choose_transfer_tpr(static_cast<int64_t>(H.p_col.size()), nc, reference_order);
        D.tpr_p = choose_transfer_tpr(static_cast<int64_t>(H.p_col.size()), n, reference_order);
        std::vector<int> po(H.p_off.begin(), H.p_off.end()), pc(H.p_col.begin(), H.p_col.end());
        std::vector<T> pv(H.p_val.size());
        for (std::size_t q = 0; q < pv.size(); ++q) pv[q] = static_cast<T>(H.p_val[q]);
        // P^T in stable fine-row order (galerkin_csr_product.h:61-80 builds the same adjacency)
        std::vector<int> to(static_cast<std::size_t>(nc) + 1, 0), tr(H.p_col.size());
        std::vector<T> tv(H.p_col.size());
        for (const uint32_t c : H.p_col) ++to[c + 1];
        for (int c = 0; c < nc; ++c) to[c + 1] += to[c];
        std::vector<int> cur(to.begin(), to.end() - 1);
        for (int i = 0; i < n; ++i)
            for (uint32_t q = H.p_off[i]; q < H.p_off[i + 1]; ++q) {
                const int pos = cur[H.p_col[q]]++;
                tr[pos] = i;
                tv[pos] = static_cast<T>(H.p_val[q]);
            }
        D.p_off.upload(po, s); D.p_col.upload(pc, s); D.p_val.upload(pv, s);
        D.r_off.upload(to, s); D.r_row.upload(tr, s); D.r_val.upload(tv, s);
        CFDXG_CUDA(cudaStreamSynchronize(s));
    }
}

// The dense coarse level's inverse, formed in FP64 from its device CSR --
// by Cholesky (cuSOLVER potrf, then potri) when the level is symmetric and
// positive definite, else by LU with partial pivoting (getrf, then getrs on
// the identity) -- and stored FP32 (or FP64 with dense_fp64).  A singular
// level fails the setup (CFDXG_ERR_SETUP).  This is set-up work (once per
// setup and per numeric refresh); the cycle applies the stored inverse with
// its own kernel.  (The earlier one-column-per-step Gauss-Jordan took 1.5 s
// at 5,287 rows: every pivot step read and wrote the whole n x 2n augmented
// matrix.)
template <class T>
void build_dense_inverse_dev(cfdxg_context* ctx, DevHierarchy<T>& d, int n, const int* ro, const int* co,
                             const double* va) {
    // under the constant null space: the inverse of the bordered matrix, of
    // which the cycle applies the leading n x n block
    const int N = n + (d.null_space ? 1 : 0);
    const std::size_t nn = static_cast<std::size_t>(n) * n;
    const std::size_t NN = static_cast<std::size_t>(N) * N;
    // the work arrays and the solver handle stay with the hierarchy for its refreshes
    DevBuf<double>& at = d.lu_a;
    DevBuf<double>& x = d.lu_x;
    at.resize(NN);
    d.lu_ipiv.resize(N);
    d.lu_info.resize(2);
    if (d.dense_fp64) d.dense64.resize(nn);
    else d.dense.resize(nn);
    cudaStream_t s = ctx->stream;
    const int64_t grid_nn = blocks_for(static_cast<int64_t>(NN), kT);
    auto init = [&] {
        CFDXG_CUDA(cudaMemsetAsync(at.get(), 0, sizeof(double) * NN, s));
        k_dense_init_t<<<blocks_for(n, kT), kT, 0, s>>>(n, N, ro, co, va, d.null_space ? 1 : 0, at.get());
        check_launch(ctx);
    };
    init();
    if (!d.solver) {
        cusolverDnHandle_t created = nullptr;
        if (cusolverDnCreate(&created) != CUSOLVER_STATUS_SUCCESS)
            throw Error(CFDXG_ERR_CUDA, "cusolverDnCreate failed");
        d.solver = std::shared_ptr<void>(created, [](void* p) { cusolverDnDestroy(static_cast<cusolverDnHandle_t>(p)); });
    }
    cusolverDnHandle_t h = static_cast<cusolverDnHandle_t>(d.solver.get());
    if (cusolverDnSetStream(h, s) != CUSOLVER_STATUS_SUCCESS) throw Error(CFDXG_ERR_CUDA, "cusolverDnSetStream failed");
    int* info = d.lu_info.get();
    int host_info[2] = {0, 0};
    // A symmetric level (no border) is inverted by Cholesky: potrf, then potri
    // on the factor -- a third of the LU route's flops (getrf, then getrs on the
    // identity).  A level that is not symmetric, or not positive definite,
    // takes the LU route.
    if (!d.null_space) {
        CFDXG_CUDA(cudaMemsetAsync(info + 1, 0, sizeof(int), s));
        k_symmetry_check<<<grid_nn, kT, 0, s>>>(N, at.get(), info + 1);
        check_launch(ctx);
        CFDXG_CUDA(cudaMemcpyAsync(&host_info[1], info + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
        CFDXG_CUDA(cudaStreamSynchronize(s));
        if (host_info[1] == 0) {
            int lw1 = 0, lw2 = 0;
            if (cusolverDnDpotrf_bufferSize(h, CUBLAS_FILL_MODE_LOWER, N, at.get(), N, &lw1) !=
                    CUSOLVER_STATUS_SUCCESS ||
                cusolverDnDpotri_bufferSize(h, CUBLAS_FILL_MODE_LOWER, N, at.get(), N, &lw2) !=
                    CUSOLVER_STATUS_SUCCESS)
                throw Error(CFDXG_ERR_CUDA, "cusolverDnDpotrf/potri_bufferSize failed");
            const int lwork = std::max({lw1, lw2, 1});
            if (static_cast<int64_t>(d.lu_work.size()) < lwork) d.lu_work.resize(static_cast<std::size_t>(lwork));
            if (cusolverDnDpotrf(h, CUBLAS_FILL_MODE_LOWER, N, at.get(), N, d.lu_work.get(), lwork, info) !=
                CUSOLVER_STATUS_SUCCESS)
                throw Error(CFDXG_ERR_CUDA, "dense coarse Cholesky failed");
            CFDXG_CUDA(cudaMemcpyAsync(&host_info[0], info, sizeof(int), cudaMemcpyDeviceToHost, s));
            CFDXG_CUDA(cudaStreamSynchronize(s));
            if (host_info[0] == 0) {
                if (cusolverDnDpotri(h, CUBLAS_FILL_MODE_LOWER, N, at.get(), N, d.lu_work.get(), lwork, info) !=
                    CUSOLVER_STATUS_SUCCESS)
                    throw Error(CFDXG_ERR_CUDA, "dense coarse Cholesky inverse failed");
                CFDXG_CUDA(cudaMemcpyAsync(&host_info[0], info, sizeof(int), cudaMemcpyDeviceToHost, s));
                if (d.dense_fp64)
                    k_dense_sym_copy<double><<<blocks_for(static_cast<int64_t>(nn), kT), kT, 0, s>>>(
                        n, N, at.get(), d.dense64.get());
                else
                    k_dense_sym_copy<float><<<blocks_for(static_cast<int64_t>(nn), kT), kT, 0, s>>>(
                        n, N, at.get(), d.dense.get());
                check_launch(ctx);
                CFDXG_CUDA(cudaStreamSynchronize(s));
                if (host_info[0] != 0)
                    throw Error(CFDXG_ERR_SETUP, "dense coarse level is singular (Cholesky inverse " +
                                                     std::to_string(host_info[0]) + ")");
                d.dense_cholesky = true;
                if (std::getenv("CFDXG_SETUP_PROFILE"))
                    std::fprintf(stderr, "[cfdxg setup] dense coarse inverse of %d rows by Cholesky\n", N);
                return;
            }
            init();   // not positive definite: the factor overwrote the matrix
        }
    }
    d.dense_cholesky = false;
    if (std::getenv("CFDXG_SETUP_PROFILE"))
        std::fprintf(stderr, "[cfdxg setup] dense coarse inverse of %d rows by LU (%s)\n", N,
                     d.null_space ? "bordered" : (host_info[1] ? "not symmetric" : "not positive definite"));
    x.resize(NN);
    k_identity<<<grid_nn, kT, 0, s>>>(N, x.get());
    check_launch(ctx);
    int lwork = 0;
    if (cusolverDnDgetrf_bufferSize(h, N, N, at.get(), N, &lwork) != CUSOLVER_STATUS_SUCCESS)
        throw Error(CFDXG_ERR_CUDA, "cusolverDnDgetrf_bufferSize failed");
    if (static_cast<int64_t>(d.lu_work.size()) < std::max(lwork, 1)) d.lu_work.resize(static_cast<std::size_t>(std::max(lwork, 1)));
    // at holds A^T column-major: factor it, then solve A^T X = I
    if (cusolverDnDgetrf(h, N, N, at.get(), N, d.lu_work.get(), d.lu_ipiv.get(), info) != CUSOLVER_STATUS_SUCCESS ||
        cusolverDnDgetrs(h, CUBLAS_OP_N, N, N, at.get(), N, d.lu_ipiv.get(), x.get(), N, info) !=
            CUSOLVER_STATUS_SUCCESS)
        throw Error(CFDXG_ERR_CUDA, "dense coarse LU failed");
    CFDXG_CUDA(cudaMemcpyAsync(&host_info[0], info, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (d.dense_fp64)
        k_dense_block_copy<double><<<blocks_for(static_cast<int64_t>(nn), kT), kT, 0, s>>>(n, N, x.get(),
                                                                                         d.dense64.get());
    else
        k_dense_block_copy<float><<<blocks_for(static_cast<int64_t>(nn), kT), kT, 0, s>>>(n, N, x.get(),
                                                                                        d.dense.get());
    check_launch(ctx);
    CFDXG_CUDA(cudaStreamSynchronize(s));
    if (host_info[0] != 0) throw Error(CFDXG_ERR_SETUP, "dense coarse level is singular (LU pivot " +
                                                            std::to_string(host_info[0]) + ")");
}

template <class T>
void build_dense_inverse(cfdxg_context* ctx, DevHierarchy<T>& d, const AmgLevel& H) {
    const int n = static_cast<int>(H.A.n);
    DevBuf<int> ro, co;
    DevBuf<double> va;
    std::vector<int> hro(H.A.ro.begin(), H.A.ro.end()), hco(H.A.co.begin(), H.A.co.end());
    ro.upload(hro, ctx->stream); co.upload(hco, ctx->stream); va.upload(H.A.va.data(), H.A.va.size(), ctx->stream);
    build_dense_inverse_dev(ctx, d, n, ro.get(), co.get(), va.get());
}

// The cycle's mean removal under the constant null space
// (amg_preconditioner.h:1310-1319); nothing without it.
template <class T, class V>
void remove_mean(cfdxg_context* ctx, DevHierarchy<T>& d, int n, V* v) {
    if (!d.null_space) return;
    const double bytes = account(3.0 * sizeof(V) * n);
    ProfScope ps(ctx, tname<T>("mean_removal_fp64", "mean_removal_fp32"), bytes);
    enqueue_remove_constant<V>(ctx->stream, n, v, d.ns_partials.get(), d.ns_in_order, true, 0.0);
    check_launch(ctx);
    count_launch(ctx);
}

template <class T>
void sweeps_from_zero(cfdxg_context* ctx, DevHierarchy<T>& d, DevLevel<T>& L, const T* r_in,
                      int sweeps) {
    cudaStream_t s = ctx->stream;
    const int gb = blocks_for(L.n, kT);
    T* x = L.x.get();
    T* x2 = L.x2.get();
    if (sweeps == 0) {
        CFDXG_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * L.n, s));
    } else {
        account(3.0 * sizeof(T) * L.n);
        launch_pdl(s, k_sweep_zero<T, T>, gb, kT, L.n, d.omega, L.inv_diag.get(), r_in, nullptr, x, d.status);
        check_launch(ctx);
        remove_mean(ctx, d, L.n, x);
        for (int k = 1; k < sweeps; ++k) {
            launch_sweep<T, T>(ctx, L, r_in, x, x2, d.omega, d.status);
            std::swap(x, x2);
            remove_mean(ctx, d, L.n, x);
        }
    }
    L.xout = x;
}

// Enqueue the cycle for levels [l, used) with the level-l right-hand side in L[l].r.
template <class T>
void enqueue_from(cfdxg_context* ctx, DevHierarchy<T>& d, int l) {
    cudaStream_t s = ctx->stream;
    DevLevel<T>& L = d.L[l];
    const int gb = blocks_for(L.n, kT);
    if (l == d.used - 1) {
        if (d.coarse_mode == 1) {
            k_dense_lu_reference<T><<<1, 32, 0, s>>>(L.n, L.ro.get(), L.co.get(), L.va.get(), L.r.get(),
                                                     L.x.get(), d.null_space ? 1 : 0, d.status);
            check_launch(ctx);
            L.xout = L.x.get();
        } else if (d.coarse_mode == 2) {
            account((d.dense_fp64 ? 8.0 : 4.0) * L.n * L.n + 2.0 * sizeof(T) * L.n);
            if (d.dense_fp64)
                launch_pdl(s, k_dense_inverse_apply<T, double>, blocks_for(static_cast<int64_t>(L.n) * 32, kT), kT,
                           L.n, d.dense64.get(), L.r.get(), L.x.get(), d.status);
            else
                launch_pdl(s, k_dense_inverse_apply<T, float>, blocks_for(static_cast<int64_t>(L.n) * 32, kT), kT,
                           L.n, d.dense.get(), L.r.get(), L.x.get(), d.status);
            check_launch(ctx);
            remove_mean(ctx, d, L.n, L.x.get());
            L.xout = L.x.get();
        } else {
            sweeps_from_zero(ctx, d, L, L.r.get(), kCoarseSweeps);
        }
        return;
    }
    if (d.coarse_pre > 0) sweeps_from_zero(ctx, d, L, L.r.get(), d.coarse_pre);
    else L.xout = L.x.get();   // x = 0: the prolongation below assigns it
    T* x = L.xout;
    T* x2 = (x == L.x.get()) ? L.x2.get() : L.x.get();
    DevLevel<T>& C = d.L[l + 1];
    if (d.coarse_pre > 0) {
        launch_residual<T>(ctx, L, L.r.get(), x, L.res.get());
        launch_restrict<T>(ctx, L, L.res.get(), C.r.get());
    } else {
        launch_restrict<T>(ctx, L, L.r.get(), C.r.get());   // x = 0: the residual is r
    }
    remove_mean(ctx, d, C.n, C.r.get());
    enqueue_from(ctx, d, l + 1);
    launch_prolong<T>(ctx, L, C.xout, x, d.status, d.coarse_pre == 0);
    remove_mean(ctx, d, L.n, x);
    for (int k = 0; k < d.coarse_post; ++k) {
        launch_sweep<T, T>(ctx, L, L.r.get(), x, x2, d.omega, d.status);
        std::swap(x, x2);
        remove_mean(ctx, d, L.n, x);
    }
    L.xout = x;
}

template <class T>
void ensure_graph(cfdxg_context* ctx, DevHierarchy<T>& d) {
    if (d.exec || d.used < 2) return;
    const int64_t before = ctx->launches;
    d.graph_bytes = 0.0;
    CFDXG_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    try {
        t_capture_bytes = &d.graph_bytes;
        enqueue_from(ctx, d, 1);
        t_capture_bytes = nullptr;
    } catch (...) {
        t_capture_bytes = nullptr;
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(ctx->stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    CFDXG_CUDA(cudaStreamEndCapture(ctx->stream, &d.graph));
    CFDXG_CUDA(cudaGraphInstantiate(&d.exec, d.graph, 0));
    d.graph_kernels = ctx->launches - before;
    ctx->launches = before;   // captured, not launched
}

}  // namespace

// FP16 fractions of each row's largest magnitude and that magnitude (the
// host upload's rounding, operation for operation).
__global__ void k_quantize_rows(int n, const int* __restrict__ ro, const double* __restrict__ va,
                                __half* __restrict__ vh, float* __restrict__ rscale) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double m = 0.0;
    for (int k = ro[i]; k < ro[i + 1]; ++k) m = fmax(m, fabs(va[k]));
    const float s = m > 0.0 ? static_cast<float>(m) : 1.0f;
    rscale[i] = s;
    for (int k = ro[i]; k < ro[i + 1]; ++k) vh[k] = __float2half_rn(static_cast<float>(va[k] / static_cast<double>(s)));
}

// The same quantisation with one warp per row, for levels with long rows (the
// row maximum is order-free, each entry's rounding is independent).
__global__ void k_quantize_rows_warp(int n, const int* __restrict__ ro, const double* __restrict__ va,
                                     __half* __restrict__ vh, float* __restrict__ rscale) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
        double m = 0.0;
        for (int k = ro[i] + lane; k < ro[i + 1]; k += 32) m = fmax(m, fabs(va[k]));
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        const float sc = m > 0.0 ? static_cast<float>(m) : 1.0f;
        if (lane == 0) rscale[i] = sc;
        for (int k = ro[i] + lane; k < ro[i + 1]; k += 32)
            vh[k] = __float2half_rn(static_cast<float>(va[k] / static_cast<double>(sc)));
    }
}

// FP16 re-quantisation of a shared-row level from FP64 values (thread or warp per row)
void quantize_level(cfdxg_context* ctx, int n, int64_t nnz, const int* ro, const double* va, __half* vh,
                    float* rscale) {
    if (nnz >= 32 * static_cast<int64_t>(n))
        k_quantize_rows_warp<<<std::max(1, std::min(blocks_for(n, 8), 148 * 32)), 256, 0, ctx->stream>>>(
            n, ro, va, vh, rscale);
    else
        k_quantize_rows<<<blocks_for(n, kT), kT, 0, ctx->stream>>>(n, ro, va, vh, rscale);
    check_launch(ctx);
}

template <class T>
__global__ void k_cast_values(int64_t n, const double* __restrict__ a, T* __restrict__ b) {
    const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) b[i] = static_cast<T>(a[i]);
}

template <class T>
void copy_or_cast(cfdxg_context* ctx, const double* src, T* dst, int64_t n) {
    if (n <= 0) return;
    if (std::is_same<T, double>::value) {
        CFDXG_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, ctx->stream));
    } else {
        k_cast_values<T><<<blocks_for(n, kT), kT, 0, ctx->stream>>>(n, src, dst);
        check_launch(ctx);
    }
}

// ---- sparsified smoothing operators (FP32 cycle, coarse_drop_tolerance)
//
// Between the fine and the coarsest level the Galerkin operators of the
// classical RS hierarchy carry many small entries (operator complexity ~27 at
// 64^3, the levels >= 1 holding 95% of the nonzeros).  The FP32 cycle's
// smoother on those levels may use a sparser operator: each row keeps its
// diagonal and the off-diagonal entries of at least theta times the row's
// largest off-diagonal magnitude, and every dropped entry is added to the
// row's diagonal (row sums, and so the constant vector's image, unchanged).
// The transfers and the coarser Galerkin operators are formed from the full
// operators as before.  A warp per row; all sums and maxima are fixed-order
// butterflies, so the result is deterministic.

// Marks the kept entries of each row (keep bits, zeroed before) and counts them.
__global__ void k_drop_mark(int n, const int* __restrict__ ro, const int* __restrict__ co,
                            const double* __restrict__ va, double theta, uint32_t* __restrict__ keep,
                            int* __restrict__ cnt) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
        const int b = ro[i], e = ro[i + 1];
        double m = 0.0;
        for (int k = b + lane; k < e; k += 32)
            if (co[k] != i) m = fmax(m, fabs(va[k]));
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        const double cut = theta * m;
        int kept = 0;
        for (int k0 = b; k0 < e; k0 += 32) {
            const int k = k0 + lane;
            const bool kp = k < e && (co[k] == i || fabs(va[k]) >= cut);
            const uint32_t bits = __ballot_sync(0xffffffffu, kp);
            kept += __popc(bits);
            if (lane == 0 && bits) {
                // the 32 entries from k0 span at most two words; rows share only their end words
                const int w = k0 >> 5, sh = k0 & 31;
                atomicOr(&keep[w], bits << sh);
                if (sh && (bits >> (32 - sh))) atomicOr(&keep[w + 1], bits >> (32 - sh));
            }
        }
        if (lane == 0) cnt[i] = kept;
    }
}

// Fills the sparsified row i from the Galerkin row and its keep bits: the
// lumped diagonal d = a_ii + sum of the dropped entries, inv_diag = 1 / d,
// the kept columns (write_columns) and values -- FP16 fractions of the kept
// row's largest magnitude (vh, rscale; the rounding of k_quantize_rows_warp)
// or T.  A zero or non-finite lumped diagonal sets the status word's
// non-finite flag.
template <class T>
__global__ void k_drop_fill(int n, const int* __restrict__ ro, const int* __restrict__ co,
                            const double* __restrict__ va, const uint32_t* __restrict__ keep,
                            const int* __restrict__ ro_s, int* __restrict__ co_s, __half* __restrict__ vh,
                            float* __restrict__ rscale, T* __restrict__ va_s, T* __restrict__ inv_diag,
                            int* status) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); i < n; i += warps) {
        const int b = ro[i], e = ro[i + 1];
        double lump = 0.0, mk = 0.0, dia = 0.0;
        for (int k = b + lane; k < e; k += 32) {
            const double v = va[k];
            if (co[k] == i) dia += v;
            else if (keep[k >> 5] >> (k & 31) & 1u) mk = fmax(mk, fabs(v));
            else lump += v;
        }
        for (int o = 16; o > 0; o >>= 1) {
            lump += __shfl_xor_sync(0xffffffffu, lump, o);
            dia += __shfl_xor_sync(0xffffffffu, dia, o);
            mk = fmax(mk, __shfl_xor_sync(0xffffffffu, mk, o));
        }
        const double d = dia + lump;
        const double m = fmax(mk, fabs(d));
        const float sc = m > 0.0 ? static_cast<float>(m) : 1.0f;
        if (lane == 0) {
            const double id = 1.0 / d;
            if (!(d != 0.0) || !isfinite(id)) atomicOr(status, kStatusNonFinite);
            inv_diag[i] = static_cast<T>(id);
            if (vh) rscale[i] = sc;
        }
        int base = ro_s[i];
        for (int k0 = b; k0 < e; k0 += 32) {
            const int k = k0 + lane;
            const bool diag = k < e && co[k] == i;
            const bool kp = k < e && (diag || (keep[k >> 5] >> (k & 31) & 1u));
            const uint32_t bits = __ballot_sync(0xffffffffu, kp);
            if (kp) {
                const int pos = base + __popc(bits & ((1u << lane) - 1u));
                const double v = diag ? d : va[k];
                if (co_s) co_s[pos] = co[k];
                if (vh) vh[pos] = __float2half_rn(static_cast<float>(v / static_cast<double>(sc)));
                else va_s[pos] = static_cast<T>(v);
            }
            base += __popc(bits);
        }
    }
}

int warp_rows_grid(int n) { return std::max(1, std::min(blocks_for(n, kT / 32), 148 * 16)); }

// Sparsifies level D from its device Galerkin operator R (setup): marks the
// kept entries, forms the row offsets and fills columns, values and inverse
// diagonal.  D keeps the keep bits for refreshes.
template <class T>
void sparsify_level(cfdxg_context* ctx, DevLevel<T>& D, const DevRefreshLevel& R, double theta, bool half) {
    cudaStream_t s = ctx->stream;
    const int n = R.n;
    D.keep.resize(static_cast<std::size_t>(std::max<int64_t>((R.nnz + 31) / 32 + 1, 1)));
    D.keep.zero(s);
    DevBuf<int> cnt(static_cast<std::size_t>(n) + 1);
    CFDXG_CUDA(cudaMemsetAsync(cnt.get() + n, 0, sizeof(int), s));
    k_drop_mark<<<warp_rows_grid(n), kT, 0, s>>>(n, R.ro.get(), R.co.get(), R.va.get(), theta, D.keep.get(),
                                                 cnt.get());
    check_launch(ctx);
    D.ro.resize(static_cast<std::size_t>(n) + 1);
    std::size_t bytes = 0;
    CFDXG_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cnt.get(), D.ro.get(), n + 1, s));
    DevBuf<unsigned char> temp(std::max<std::size_t>(bytes, 1));
    CFDXG_CUDA(cub::DeviceScan::ExclusiveSum(temp.get(), bytes, cnt.get(), D.ro.get(), n + 1, s));
    int nnz = 0;
    CFDXG_CUDA(cudaMemcpyAsync(&nnz, D.ro.get() + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    CFDXG_CUDA(cudaStreamSynchronize(s));
    D.nnz = nnz;
    D.narrow = false;
    D.co16.release();
    D.co.resize(static_cast<std::size_t>(std::max(nnz, 1)));
    D.half = half;
    if (half) {
        D.vh.resize(static_cast<std::size_t>(std::max(nnz, 1)));
        D.rscale.resize(static_cast<std::size_t>(n));
        D.va.release();
    } else {
        D.va.resize(static_cast<std::size_t>(std::max(nnz, 1)));
        D.vh.release();
        D.rscale.release();
    }
    D.inv_diag.resize(static_cast<std::size_t>(n));
    D.sparsified = true;
}

// (Re-)forms the sparsified level's values and inverse diagonal from the
// Galerkin values R.va (setup and numeric refresh; the kept pattern is fixed).
template <class T>
void fill_sparsified(cfdxg_context* ctx, DevLevel<T>& D, const DevRefreshLevel& R, bool columns) {
    __half* vh = nullptr;
    float* rs = nullptr;
    if constexpr (std::is_same<T, float>::value) {
        if (D.half) { vh = D.vh.get(); rs = D.rscale.get(); }
    }
    k_drop_fill<T><<<warp_rows_grid(R.n), kT, 0, ctx->stream>>>(
        R.n, R.ro.get(), R.co.get(), R.va.get(), D.keep.get(), D.ro.get(), columns ? D.co.get() : nullptr, vh, rs,
        D.half ? nullptr : D.va.get(), D.inv_diag.get(), ctx->scratch.status);
    check_launch(ctx);
}

// ---- the same upload from the device copy the setup's Galerkin products left

// flag = 1 when some |column - row| does not fit in 16 bits
__global__ void k_narrow_check(int n, const int* __restrict__ ro, const int* __restrict__ co, int* flag) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = ro[i]; k < ro[i + 1]; ++k) {
        const int d = co[k] - i;
        if (d < INT16_MIN || d > INT16_MAX) { atomicOr(flag, 1); return; }
    }
}

__global__ void k_narrow_columns(int n, const int* __restrict__ ro, const int* __restrict__ co,
                                 int16_t* __restrict__ c16) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int k = ro[i]; k < ro[i + 1]; ++k) c16[k] = static_cast<int16_t>(co[k] - i);
}

// P^T values in the stable fine-row order of the setup's P^T adjacency
template <class T>
__global__ void k_transpose_values(int64_t m, const int* __restrict__ t_row, const int* __restrict__ t_pos,
                                   const int* __restrict__ p_off, const double* __restrict__ p_val,
                                   T* __restrict__ r_val) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < m) r_val[t] = static_cast<T>(p_val[p_off[t_row[t]] + t_pos[t]]);
}

template <class T>
void device_copy(cfdxg_context* ctx, DevBuf<T>& dst, const T* src, int64_t count) {
    dst.resize(static_cast<std::size_t>(std::max<int64_t>(count, 1)));
    if (count > 0)
        CFDXG_CUDA(cudaMemcpyAsync(dst.get(), src, sizeof(T) * count, cudaMemcpyDeviceToDevice, ctx->stream));
}

template <class T>
void upload_transfers_device(cfdxg_context* ctx, DevLevel<T>& D, const AmgLevel& H, const DevRefreshLevel& R,
                             const UploadOptions& opt);

// upload_level from the setup's device level (int CSR, FP64 values, P and the
// stable P^T adjacency): the same layout choices and the same values, formed
// by kernels instead of host loops.
template <class T>
void upload_level_device(cfdxg_context* ctx, DevLevel<T>& D, const AmgLevel& H, const DevRefreshLevel& R,
                         bool with_transfer, const UploadOptions& opt, bool sparsify) {
    cudaStream_t s = ctx->stream;
    D.n = R.n;
    D.nnz = static_cast<int>(R.nnz);
    if (sparsify) {
        sparsify_level(ctx, D, R, opt.coarse_drop_tolerance, std::is_same<T, float>::value && opt.half_values);
        D.tpr = choose_sparse_tpr(D.nnz, D.n);
        fill_sparsified(ctx, D, R, true);
        upload_transfers_device(ctx, D, H, R, opt);
        D.r.resize(D.n); D.x.resize(D.n); D.x2.resize(D.n); D.res.resize(D.n);
        CFDXG_CUDA(cudaStreamSynchronize(s));
        return;
    }
    D.tpr = choose_tpr(D.nnz, D.n, opt.reference_order);
    device_copy(ctx, D.ro, R.ro.get(), D.n + 1);
    bool narrow = with_transfer && opt.narrow_columns && D.tpr == 1;
    if (narrow) {
        DevBuf<int> flag(1);
        flag.zero(s);
        k_narrow_check<<<blocks_for(D.n, kT), kT, 0, s>>>(D.n, R.ro.get(), R.co.get(), flag.get());
        check_launch(ctx);
        int h = 0;
        CFDXG_CUDA(cudaMemcpyAsync(&h, flag.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        CFDXG_CUDA(cudaStreamSynchronize(s));
        narrow = h == 0;
    }
    D.narrow = narrow;
    if (narrow) {
        D.co16.resize(static_cast<std::size_t>(std::max(D.nnz, 1)));
        k_narrow_columns<<<blocks_for(D.n, kT), kT, 0, s>>>(D.n, R.ro.get(), R.co.get(), D.co16.get());
        check_launch(ctx);
        D.co.release();
    } else {
        device_copy(ctx, D.co, R.co.get(), D.nnz);
        D.co16.release();
    }
    D.half = std::is_same<T, float>::value && opt.half_values && with_transfer && D.tpr > 1;
    if (D.half) {
        if constexpr (std::is_same<T, float>::value) {
            D.vh.resize(static_cast<std::size_t>(std::max(D.nnz, 1)));
            D.rscale.resize(static_cast<std::size_t>(D.n));
            quantize_level(ctx, D.n, R.nnz, R.ro.get(), R.va.get(), D.vh.get(), D.rscale.get());
        }
        D.va.release();
    } else {
        D.va.resize(static_cast<std::size_t>(std::max(D.nnz, 1)));
        copy_or_cast<T>(ctx, R.va.get(), D.va.get(), D.nnz);
    }
    std::vector<T> d(H.inv_diag.size());
    for (std::size_t k = 0; k < d.size(); ++k) d[k] = static_cast<T>(H.inv_diag[k]);
    D.inv_diag.upload(d, s);
    D.r.resize(D.n); D.x.resize(D.n); D.x2.resize(D.n); D.res.resize(D.n);
    if (with_transfer) upload_transfers_device(ctx, D, H, R, opt);
    CFDXG_CUDA(cudaStreamSynchronize(s));
}

// P and P^T of a level from the setup's device copy
template <class T>
void upload_transfers_device(cfdxg_context* ctx, DevLevel<T>& D, const AmgLevel& H, const DevRefreshLevel& R,
                             const UploadOptions& opt) {
    cudaStream_t s = ctx->stream;
    {
        const int64_t pn = static_cast<int64_t>(H.p_col.size());
        D.nc = R.n_coarse;
        D.tpr_r = choose_transfer_tpr(pn, D.nc, opt.reference_order);
        D.tpr_p = choose_transfer_tpr(pn, D.n, opt.reference_order);
        device_copy(ctx, D.p_off, R.p_off.get(), D.n + 1);
        device_copy(ctx, D.p_col, R.p_col.get(), pn);
        D.p_val.resize(static_cast<std::size_t>(std::max<int64_t>(pn, 1)));
        copy_or_cast<T>(ctx, R.p_val.get(), D.p_val.get(), pn);
        device_copy(ctx, D.r_off, R.t_off.get(), D.nc + 1);
        device_copy(ctx, D.r_row, R.t_row.get(), pn);
        D.r_val.resize(static_cast<std::size_t>(std::max<int64_t>(pn, 1)));
        if (pn > 0) {
            k_transpose_values<T><<<blocks_for(pn, kT), kT, 0, s>>>(pn, R.t_row.get(), R.t_pos.get(), R.p_off.get(),
                                                                    R.p_val.get(), D.r_val.get());
            check_launch(ctx);
        }
    }
    CFDXG_CUDA(cudaStreamSynchronize(s));
}

template <class T>
std::unique_ptr<DevHierarchy<T>> upload_hierarchy(cfdxg_context* ctx, const AmgHierarchy& h,
                                                  const UploadOptions& opt, const DevRefresh* R) {
    const int coarse_dense_limit = opt.coarse_dense_limit;
    auto d = std::make_unique<DevHierarchy<T>>();
    d->omega = static_cast<T>(h.omega);
    d->pre = h.options.pre;
    d->post = h.options.post;
    // Levels >= 1: the reference's pre/post counts for the FP64 cycle.  The FP32
    // cycle defaults to one post-sweep and no pre-sweep there (its fine level
    // keeps pre/post): the coarse operators hold ~25x the fine level's nonzeros,
    // and V(0,1) reads each of them once per cycle instead of twice for V(1,1).
    const bool fp32 = std::is_same<T, float>::value;
    const int coarse_default_pre = fp32 ? kFp32CoarsePre : h.options.pre;
    const int coarse_default_post = fp32 ? kFp32CoarsePost : h.options.post;
    d->coarse_pre = h.options.coarse_pre >= 0 ? h.options.coarse_pre : coarse_default_pre;
    d->coarse_post = h.options.coarse_post >= 0 ? h.options.coarse_post : coarse_default_post;
    d->status = ctx->scratch.status;
    d->dense_fp64 = opt.dense_fp64;
    d->null_space = opt.constant_null_space;
    d->ns_in_order = opt.reference_order;
    if (d->null_space) d->ns_partials.resize(kNsMaxBlocks);
    int used = static_cast<int>(h.levels.size());
    d->coarse_mode = 0;
    if (std::is_same<T, float>::value && coarse_dense_limit > 0) {
        for (int l = 0; l < used; ++l)
            if (h.levels[l].A.n <= coarse_dense_limit) { used = l + 1; d->coarse_mode = 2; break; }
    }
    if (d->coarse_mode == 0 && h.levels[used - 1].A.n <= kDenseDirectLimit) d->coarse_mode = 1;
    d->used = used;
    d->L.resize(used);
    // from the setup's device copy of the levels when there is one
    const bool from_device = R && static_cast<int>(R->L.size()) >= used;
    for (int l = 0; l < used; ++l) {
        // the FP32 cycle's smoothing operators between the fine and the coarsest level
        const bool sparsify = fp32 && opt.coarse_drop_tolerance > 0.0 && !opt.reference_order && l >= 1 &&
                              l + 1 < used;
        if (from_device) upload_level_device(ctx, d->L[l], h.levels[l], R->L[l], l + 1 < used, opt, sparsify);
        else upload_level(ctx, d->L[l], h.levels[l], l + 1 < used, opt);
    }
    if (d->coarse_mode == 2) {
        if (from_device) {
            const DevRefreshLevel& C = R->L[used - 1];
            build_dense_inverse_dev(ctx, *d, C.n, C.ro.get(), C.co.get(), C.va.get());
        } else {
            build_dense_inverse(ctx, *d, h.levels[used - 1]);
        }
    }
    return d;
}

// New level values, inverse diagonals and damping from the device refresh
// (the transfer operators and every pattern are unchanged).
template <class T>
void set_hierarchy_values_device(cfdxg_context* ctx, DevHierarchy<T>& d, const DevRefresh& R, double omega) {
    d.omega = static_cast<T>(omega);
    for (int l = 0; l < d.used; ++l) {
        if (d.L[l].sparsified) {
            fill_sparsified(ctx, d.L[l], R.L[l], false);
            continue;
        }
        if (d.L[l].half) {
            if constexpr (std::is_same<T, float>::value)
                quantize_level(ctx, d.L[l].n, R.L[l].nnz, d.L[l].ro.get(), R.L[l].va.get(), d.L[l].vh.get(),
                               d.L[l].rscale.get());
        } else {
            copy_or_cast<T>(ctx, R.L[l].va.get(), d.L[l].va.get(), R.L[l].nnz);
        }
        copy_or_cast<T>(ctx, R.L[l].inv_diag.get(), d.L[l].inv_diag.get(), R.L[l].n);
    }
    if (d.coarse_mode == 2) {
        ProfScope ps(ctx, "refresh_dense_inverse", 0.0);
        const DevRefreshLevel& C = R.L[d.used - 1];
        build_dense_inverse_dev(ctx, d, C.n, C.ro.get(), C.co.get(), C.va.get());
    }
    // omega is a kernel argument baked into the graph: recapture
    if (d.exec) { cudaGraphExecDestroy(d.exec); d.exec = nullptr; }
    if (d.graph) { cudaGraphDestroy(d.graph); d.graph = nullptr; }
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
}

template <class T>
void vcycle_apply(cfdxg_context* ctx, DevHierarchy<T>& d, const double* r, double* z) {
    cudaStream_t s = ctx->stream;
    DevLevel<T>& L = d.L[0];
    const int gb = blocks_for(L.n, kT);
    if (d.used == 1) {
        // single-level hierarchy: the coarsest treatment applies to the fine level
        launch_pdl(s, k_copy_cast<double, T>, gb, kT, L.n, r, L.r.get());
        check_launch(ctx);
        remove_mean(ctx, d, L.n, L.r.get());
        enqueue_from(ctx, d, 0);
        launch_pdl(s, k_copy_cast<T, double>, gb, kT, L.n, L.xout, z);
        check_launch(ctx);
        remove_mean(ctx, d, L.n, z);
        return;
    }
    ensure_graph(ctx, d);
    // Level-0 right-hand side: FP64 reads the caller's r directly; FP32 converts
    // it in the first sweep.  Under the constant null space both first copy it
    // and remove its mean (the compatible right-hand side of apply()).
    const T* rl = nullptr;
    T* x = L.x.get();
    T* x2 = L.x2.get();
    const bool own_copy = d.null_space || !std::is_same<T, double>::value;
    if (d.null_space) {
        launch_pdl(s, k_copy_cast<double, T>, gb, kT, L.n, r, L.r.get());
        check_launch(ctx);
        remove_mean(ctx, d, L.n, L.r.get());
    }
    rl = own_copy ? L.r.get() : reinterpret_cast<const T*>(r);
    if (d.pre == 0) {
        if (!std::is_same<T, double>::value && !d.null_space) {
            launch_pdl(s, k_copy_cast<double, T>, gb, kT, L.n, r, L.r.get());
            check_launch(ctx);
        }
        CFDXG_CUDA(cudaMemsetAsync(x, 0, sizeof(T) * L.n, s));
    } else {
        if (d.null_space)
            launch_pdl(s, k_sweep_zero<T, T>, gb, kT, L.n, d.omega, L.inv_diag.get(), rl, nullptr, x, d.status);
        else
            launch_pdl(s, k_sweep_zero<T, double>, gb, kT, L.n, d.omega, L.inv_diag.get(), r,
                       std::is_same<T, double>::value ? nullptr : L.r.get(), x, d.status);
        check_launch(ctx);
        remove_mean(ctx, d, L.n, x);
        for (int k = 1; k < d.pre; ++k) {
            launch_sweep<T, T>(ctx, L, rl, x, x2, d.omega, d.status);
            std::swap(x, x2);
            remove_mean(ctx, d, L.n, x);
        }
    }
    launch_residual<T>(ctx, L, rl, x, L.res.get());
    DevLevel<T>& C = d.L[1];
    launch_restrict<T>(ctx, L, L.res.get(), C.r.get());
    remove_mean(ctx, d, C.n, C.r.get());
    {
        ProfScope ps(ctx, tname<T>("vcycle_levels_1plus_fp64_graph", "vcycle_levels_1plus_fp32_graph"), d.graph_bytes);
        CFDXG_CUDA(cudaGraphLaunch(d.exec, s));
    }
    count_launch(ctx, d.graph_kernels);
    launch_prolong<T>(ctx, L, C.xout, x, d.status);
    remove_mean(ctx, d, L.n, x);
    if (d.post == 0) {
        launch_pdl(s, k_copy_cast<T, double>, gb, kT, L.n, x, z);
        check_launch(ctx);
        remove_mean(ctx, d, L.n, z);
        return;
    }
    for (int k = 0; k < d.post; ++k) {
        if (k + 1 == d.post) {
            launch_sweep<T, double>(ctx, L, rl, x, z, d.omega, d.status);
            remove_mean(ctx, d, L.n, z);
        } else {
            launch_sweep<T, T>(ctx, L, rl, x, x2, d.omega, d.status);
            std::swap(x, x2);
            remove_mean(ctx, d, L.n, x);
        }
    }
    remove_mean(ctx, d, L.n, z);   // apply()'s removal from the result
}

template <class T>
void destroy_hierarchy(DevHierarchy<T>* d) { delete d; }

template std::unique_ptr<DevHierarchy<double>> upload_hierarchy<double>(cfdxg_context*, const AmgHierarchy&, const UploadOptions&,
                                                                         const DevRefresh*);
template std::unique_ptr<DevHierarchy<float>> upload_hierarchy<float>(cfdxg_context*, const AmgHierarchy&, const UploadOptions&,
                                                                       const DevRefresh*);
template void set_hierarchy_values_device<double>(cfdxg_context*, DevHierarchy<double>&, const DevRefresh&, double);
template void set_hierarchy_values_device<float>(cfdxg_context*, DevHierarchy<float>&, const DevRefresh&, double);
template void vcycle_apply<double>(cfdxg_context*, DevHierarchy<double>&, const double*, double*);
template void vcycle_apply<float>(cfdxg_context*, DevHierarchy<float>&, const double*, double*);
template void destroy_hierarchy<double>(DevHierarchy<double>*);
template void destroy_hierarchy<float>(DevHierarchy<float>*);

}  // namespace cfdxg
