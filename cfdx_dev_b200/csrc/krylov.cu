// krylov.cu -- device-resident right-preconditioned GMRES / FGMRES.
//
// Restates solve_gmres (core/linalg/gmres_solver.h:28-600) with its exact
// control flow: two-pass modified Gram-Schmidt, scaled two-pass norms
// (krylov_norm2, core/linalg/krylov_reductions.h:84-115), Givens rotations,
// Arnoldi/Hessenberg breakdown floors, periodic residual-replacement checks,
// adaptive restart (krylov_controls.h:28-51), best-iterate retention, the
// b = 0 shifted solve, and stored Z (so variable preconditioners are valid).
//
// Vectors (basis V, preconditioned basis Z, x, r, w) live on the device; each
// Arnoldi step ends with one small device->host copy of its Hessenberg column
// and norms, and the host runs the same scalar Givens / least-squares code as
// the reference.  Dots and norms are deterministic: a fixed partition into
// blocks (it depends only on n), a fixed in-block tree and an in-order final
// sum, so repeated solves are bitwise identical.
#include <algorithm>
#include <cmath>
#include <functional>
#include <limits>
#include <mutex>
#include <type_traits>

#include "krylov.h"
#include "nullspace.cuh"

namespace cfdxg {

namespace {

constexpr int kT = kReduceThreads;
constexpr double kEps = std::numeric_limits<double>::epsilon();

// scalar slots in ctx->scratch.scalars
enum Slot : int {
    kMax = 0, kInvalid = 1, kNorm = 2, kDot = 3, kBeta = 4, kHnext = 5, kAction = 6,
    kH1 = 64, kH2 = 64 + 1024, kY = 64 + 2048, kSlots = 4096
};

__global__ void k_absmax(int n, const double* __restrict__ a, double* partial, unsigned* ticket,
                         double* out_max, double* out_invalid) {
    pdl_entry();
    __shared__ double sm[32];
    double m = 0.0, bad = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double v = a[i];
        if (!isfinite(v)) bad = 1.0;
        m = fmax(m, fabs(v));
    }
    m = block_max(m, sm);
    bad = block_max(bad, sm);
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = m; partial[2 * blockIdx.x + 1] = bad; }
    if (last_block(ticket)) {
        double mm = 0.0, bb = 0.0;
        for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
            mm = fmax(mm, partial[2 * b]);
            bb = fmax(bb, partial[2 * b + 1]);
        }
        mm = block_max(mm, sm);
        bb = block_max(bb, sm);
        if (threadIdx.x == 0) { *out_max = mm; *out_invalid = bb; *ticket = 0; }
    }
}

// out = scale * sqrt(sum (a_i / scale)^2), NaN on invalid input, 0 when scale == 0.
__global__ void k_sumsq(int n, const double* __restrict__ a, const double* scale_p,
                        const double* invalid_p, double* partial, unsigned* ticket, double* out) {
    pdl_entry();
    __shared__ double sm[32];
    const double scale = *scale_p;
    double s = 0.0;
    if (scale > 0.0)
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
            const double q = a[i] / scale;
            s += q * q;
        }
    s = block_sum(s, sm);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
    if (last_block(ticket)) {
        double t = 0.0;
        for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) t += partial[b];
        t = block_sum(t, sm);
        if (threadIdx.x == 0) {
            double r;
            if (*invalid_p > 0.0) r = nan("");
            else if (scale == 0.0) r = 0.0;
            else if (!isfinite(t)) r = nan("");
            else r = scale * sqrt(fmax(0.0, t));
            *out = r;
            *ticket = 0;
        }
    }
}

__global__ void k_dot(int n, const double* __restrict__ a, const double* __restrict__ b, double* partial,
                      unsigned* ticket, double* out) {
    pdl_entry();
    __shared__ double sm[32];
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += a[i] * b[i];
    s = block_sum(s, sm);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
    if (last_block(ticket)) {
        double t = 0.0;
        for (int q = threadIdx.x; q < gridDim.x; q += blockDim.x) t += partial[q];
        t = block_sum(t, sm);
        if (threadIdx.x == 0) { *out = t; *ticket = 0; }
    }
}

// Modified Gram-Schmidt step fused with the next step's dot: w = w - c v
// (k_axpy_neg's arithmetic), then out = sum_i u_i w_i over the updated w with
// k_dot's partition and order -- bit-identical to the two kernels in turn,
// one pass over w instead of two.
__global__ void k_axpy_dot(int n, double* __restrict__ w, const double* __restrict__ v, const double* c,
                           const double* __restrict__ u, double* partial, unsigned* ticket, double* out) {
    pdl_entry();
    __shared__ double sm[32];
    const double cc = *c;
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double wi = w[i] - cc * v[i];
        w[i] = wi;
        s += u[i] * wi;
    }
    s = block_sum(s, sm);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
    if (last_block(ticket)) {
        double t = 0.0;
        for (int q = threadIdx.x; q < gridDim.x; q += blockDim.x) t += partial[q];
        t = block_sum(t, sm);
        if (threadIdx.x == 0) { *out = t; *ticket = 0; }
    }
}

// The last Gram-Schmidt step fused with the first pass of the norm: w = w - c v,
// then k_absmax over the updated w.
__global__ void k_axpy_absmax(int n, double* __restrict__ w, const double* __restrict__ v, const double* c,
                              double* partial, unsigned* ticket, double* out_max, double* out_invalid) {
    pdl_entry();
    __shared__ double sm[32];
    const double cc = *c;
    double m = 0.0, bad = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double wi = w[i] - cc * v[i];
        w[i] = wi;
        if (!isfinite(wi)) bad = 1.0;
        m = fmax(m, fabs(wi));
    }
    m = block_max(m, sm);
    bad = block_max(bad, sm);
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = m; partial[2 * blockIdx.x + 1] = bad; }
    if (last_block(ticket)) {
        double mm = 0.0, bb = 0.0;
        for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
            mm = fmax(mm, partial[2 * b]);
            bb = fmax(bb, partial[2 * b + 1]);
        }
        mm = block_max(mm, sm);
        bb = block_max(bb, sm);
        if (threadIdx.x == 0) { *out_max = mm; *out_invalid = bb; *ticket = 0; }
    }
}

// ---- classical Gram-Schmidt (the CGS2 option): up to kChunk basis vectors per launch
constexpr int kChunk = 16;
// The multi-vector passes take the same fixed grid of eight blocks per SM as
// the single-vector reductions (the reduction partition, so deterministic).
constexpr int kWideBlocks = kMaxReduceBlocks;

// out[q] = v_{i0+q} . w for q < c, one pass over w.  Each block's partial sums
// land in partial[q * gridDim.x + block]; the last block adds them in block
// order (deterministic, as k_dot).
__global__ void k_multidot(int n, const double* __restrict__ V, int i0, int c, const double* __restrict__ w,
                           double* partial, unsigned* ticket, double* out) {
    pdl_entry();
    __shared__ double sm[32];
    double acc[kChunk];
#pragma unroll
    for (int q = 0; q < kChunk; ++q) acc[q] = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const double wk = w[k];
#pragma unroll
        for (int q = 0; q < kChunk; ++q)
            if (q < c) acc[q] += V[static_cast<size_t>(i0 + q) * n + k] * wk;
    }
#pragma unroll
    for (int q = 0; q < kChunk; ++q) {
        if (q >= c) break;
        const double s = block_sum(acc[q], sm);
        if (threadIdx.x == 0) partial[q * gridDim.x + blockIdx.x] = s;
    }
    if (last_block(ticket)) {
        for (int q = 0; q < c; ++q) {
            double t = 0.0;
            for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) t += partial[q * gridDim.x + b];
            t = block_sum(t, sm);
            if (threadIdx.x == 0) out[q] = t;
        }
        if (threadIdx.x == 0) *ticket = 0;
    }
}

// w -= sum_{q<c} h[q] v_{i0+q}, subtracting in q order per element; with
// absmax, also the first pass of the norm of the updated w (as k_absmax).
template <bool ABSMAX>
__global__ void k_multi_axpy(int n, const double* __restrict__ V, int i0, int c, const double* h,
                             double* __restrict__ w, double* partial, unsigned* ticket, double* out_max,
                             double* out_invalid) {
    pdl_entry();
    __shared__ double sm[32];
    __shared__ double hs[kChunk];
    if (threadIdx.x < c) hs[threadIdx.x] = h[threadIdx.x];
    __syncthreads();
    double m = 0.0, bad = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double wk = w[k];
#pragma unroll
        for (int q = 0; q < kChunk; ++q)
            if (q < c) wk = wk - hs[q] * V[static_cast<size_t>(i0 + q) * n + k];
        w[k] = wk;
        if (ABSMAX) {
            if (!isfinite(wk)) bad = 1.0;
            m = fmax(m, fabs(wk));
        }
    }
    if (!ABSMAX) return;
    m = block_max(m, sm);
    bad = block_max(bad, sm);
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = m; partial[2 * blockIdx.x + 1] = bad; }
    if (last_block(ticket)) {
        double mm = 0.0, bb = 0.0;
        for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
            mm = fmax(mm, partial[2 * b]);
            bb = fmax(bb, partial[2 * b + 1]);
        }
        mm = block_max(mm, sm);
        bb = block_max(bb, sm);
        if (threadIdx.x == 0) { *out_max = mm; *out_invalid = bb; *ticket = 0; }
    }
}

// ---- fused classical Gram-Schmidt passes (the CGS2 option, at most kChunk
// basis vectors): three passes over the basis per Arnoldi step instead of
// four, and the two norms of w taken inside them (plain sums of squares: this
// option is the library's own orthogonalisation, not the reference's MGS2).
// Each pass runs one resident wave (the blocks of its instance that fit on
// the GPU at once: a partition that depends only on n, the basis count and
// the GPU, so the sums are deterministic) and reduces all outputs at once:
// per warp by a fixed butterfly, per block in warp order, and over the
// blocks by one warp per output in a fixed lane/butterfly order.
constexpr int kGsWarps = kT / 32;

// out[q] = grid sum of acc[q] for q < C; with EXTRA also out[C] = grid sum of extra.
template <int C, bool EXTRA>
__device__ __forceinline__ void grid_multi_sum(const double (&acc)[C], double extra, double* partial,
                                               unsigned* ticket, double* out) {
    constexpr int kOut = C + (EXTRA ? 1 : 0);
    __shared__ double wsum[kGsWarps][kOut];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < C; ++q) {
        double v = acc[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) wsum[warp][q] = v;
    }
    if (EXTRA) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) extra += __shfl_xor_sync(0xffffffffu, extra, o);
        if (lane == 0) wsum[warp][kOut - 1] = extra;
    }
    __syncthreads();
    if (threadIdx.x < kOut) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < kGsWarps; ++w) t += wsum[w][threadIdx.x];
        partial[threadIdx.x * gridDim.x + blockIdx.x] = t;
    }
    if (last_block(ticket)) {
        for (int q = warp; q < kOut; q += kGsWarps) {
            double t = 0.0;
            for (int b = lane; b < static_cast<int>(gridDim.x); b += 32) t += partial[q * gridDim.x + b];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == 0) out[q] = t;
        }
        if (threadIdx.x == 0) *ticket = 0;
    }
}

// The fused passes are instantiated for each basis count C (1..kChunk): the
// per-vector accumulators and loads take exactly C registers' worth, so the
// small counts of the first Arnoldi steps run at higher occupancy.

// out[q] = v_q . w for q < C, and out[C] = w . w (the Arnoldi action norm squared)
template <int C>
__global__ void __launch_bounds__(kT) k_gs_first(int n, const double* __restrict__ V,
                                                 const double* __restrict__ w, double* partial, unsigned* ticket,
                                                 double* out) {
    pdl_entry();
    double acc[C];
#pragma unroll
    for (int q = 0; q < C; ++q) acc[q] = 0.0;
    double ww = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const double wk = w[k];
#pragma unroll
        for (int q = 0; q < C; ++q) acc[q] += V[static_cast<size_t>(q) * n + k] * wk;
        ww += wk * wk;
    }
    grid_multi_sum<C, true>(acc, ww, partial, ticket, out);
}

// w -= sum_{q<C} h[q] v_q (in q order per element), then out[q] = v_q . w over the updated w
template <int C>
__global__ void __launch_bounds__(kT) k_gs_axpy_dot(int n, const double* __restrict__ V, const double* h,
                                                    double* __restrict__ w, double* partial, unsigned* ticket,
                                                    double* out) {
    pdl_entry();
    __shared__ double hs[C];
    if (threadIdx.x < C) hs[threadIdx.x] = h[threadIdx.x];
    __syncthreads();
    double acc[C];
#pragma unroll
    for (int q = 0; q < C; ++q) acc[q] = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double vk[C];
        double wk = w[k];
#pragma unroll
        for (int q = 0; q < C; ++q) {
            vk[q] = V[static_cast<size_t>(q) * n + k];
            wk = wk - hs[q] * vk[q];
        }
        w[k] = wk;
#pragma unroll
        for (int q = 0; q < C; ++q) acc[q] += vk[q] * wk;
    }
    grid_multi_sum<C, false>(acc, 0.0, partial, ticket, out);
}

// w -= sum_{q<C} h[q] v_q, then *norm_out = sqrt(w . w) (NaN when not finite)
template <int C>
__global__ void k_gs_axpy_norm(int n, const double* __restrict__ V, const double* h, double* __restrict__ w,
                               double* partial, unsigned* ticket, double* norm_out) {
    pdl_entry();
    __shared__ double sm[32];
    __shared__ double hs[C];
    if (threadIdx.x < C) hs[threadIdx.x] = h[threadIdx.x];
    __syncthreads();
    double ss = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        double wk = w[k];
#pragma unroll
        for (int q = 0; q < C; ++q) wk = wk - hs[q] * V[static_cast<size_t>(q) * n + k];
        w[k] = wk;
        ss += wk * wk;
    }
    ss = block_sum(ss, sm);
    if (threadIdx.x == 0) partial[blockIdx.x] = ss;
    if (last_block(ticket)) {
        double t = 0.0;
        for (int b = threadIdx.x; b < gridDim.x; b += blockDim.x) t += partial[b];
        t = block_sum(t, sm);
        if (threadIdx.x == 0) {
            *norm_out = isfinite(t) ? sqrt(t) : nan("");
            *ticket = 0;
        }
    }
}

// Blocks of kT threads of the kernel K resident on one SM (cached per kernel
// instance: the answer depends only on the binary and the architecture).
template <auto K>
int resident_per_sm() {
    static const int per_sm = [] {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, K, kT, 0) != cudaSuccess) b = 1;
        return std::max(1, b);
    }();
    return per_sm;
}

// Calls go(std::integral_constant<int, C>) for the basis count c in 1..kChunk.
template <class Go>
void with_basis_count(int c, Go&& go) {
    switch (c) {
#define CFDXG_GS_CASE(C) case C: go(std::integral_constant<int, C>{}); break;
        CFDXG_GS_CASE(1) CFDXG_GS_CASE(2) CFDXG_GS_CASE(3) CFDXG_GS_CASE(4) CFDXG_GS_CASE(5) CFDXG_GS_CASE(6)
        CFDXG_GS_CASE(7) CFDXG_GS_CASE(8) CFDXG_GS_CASE(9) CFDXG_GS_CASE(10) CFDXG_GS_CASE(11)
        CFDXG_GS_CASE(12) CFDXG_GS_CASE(13) CFDXG_GS_CASE(14) CFDXG_GS_CASE(15) CFDXG_GS_CASE(16)
#undef CFDXG_GS_CASE
        default: throw Error(CFDXG_ERR_INVALID_ARGUMENT, "Gram-Schmidt basis count out of range");
    }
}

// w = w - c * v   (gmres_solver.h:283 / :289)
__global__ void k_axpy_neg(int n, double* __restrict__ w, const double* __restrict__ v, const double* c) {
    pdl_entry();
    const double cc = *c;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) w[i] = w[i] - cc * v[i];
}

// v = w / d  when d > 0   (gmres_solver.h:183 and :322)
__global__ void k_div(int n, const double* __restrict__ w, const double* d, double* __restrict__ v) {
    pdl_entry();
    const double dd = *d;
    if (!(dd > 0.0)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = w[i] / dd;
}

// r = b - A x  (true residual with the FP64 operator)
__global__ void k_true_residual(int n, const int* __restrict__ ro, const int* __restrict__ co,
                                const double* __restrict__ va, const double* __restrict__ b,
                                const double* __restrict__ x, double* __restrict__ r) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    const int e = ro[i + 1];
    for (int k = ro[i]; k < e; ++k) s += va[k] * __ldg(x + co[k]);
    r[i] = b[i] - s;
}

// out = x + sum_j y_j z_j, accumulated in j order per element (gmres_solver.h:497-501)
__global__ void k_update(int n, const double* __restrict__ x, const double* __restrict__ Z,
                         const double* __restrict__ y, int used, double* __restrict__ out) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = x[i];
    for (int j = 0; j < used; ++j) v += y[j] * Z[static_cast<size_t>(j) * n + i];
    out[i] = v;
}

// *to = sqrt(*from) (NaN when *from is not finite)
__global__ void k_sqrt_slot(const double* from, double* to) {
    const double v = *from;
    *to = isfinite(v) ? sqrt(v) : nan("");
}

__global__ void k_neg(int n, const double* __restrict__ a, double* __restrict__ b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = -a[i];
}

__global__ void k_add(int n, double* __restrict__ x, const double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += y[i];
}

// r = b - y
__global__ void k_sub(int n, const double* __restrict__ b, const double* __restrict__ y, double* __restrict__ r) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = b[i] - y[i];
}

__global__ void k_fill(int n, double v, double* __restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = v;
}

// y = A^T x (column sums of a_ij x_i; the order of the additions varies with
// scheduling -- used only for the threshold of is_bilateral_null_space)
__global__ void k_transpose_apply(int n, const int* __restrict__ ro, const int* __restrict__ co,
                                  const double* __restrict__ va, const double* __restrict__ x,
                                  double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double xi = x[i];
    for (int k = ro[i]; k < ro[i + 1]; ++k) atomicAdd(y + co[k], va[k] * xi);
}

// Pinned copies of one Arnoldi step's scalar slots [0, kH2 + m + 1) and of
// the status word, two of them (step j uses buffer j & 1), each with the
// event that marks its copy done: the host reads step j's results while the
// GPU runs step j + 1.
struct StepMirror {
    double* scalars[2] = {nullptr, nullptr};
    int* status[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    StepMirror() {
        for (int k = 0; k < 2; ++k) {
            CFDXG_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&scalars[k]), sizeof(double) * kSlots,
                                     cudaHostAllocDefault));
            CFDXG_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&status[k]), sizeof(int), cudaHostAllocDefault));
            CFDXG_CUDA(cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming));
        }
    }
    ~StepMirror() {
        for (int k = 0; k < 2; ++k) {
            if (scalars[k]) cudaFreeHost(scalars[k]);
            if (status[k]) cudaFreeHost(status[k]);
            if (done[k]) cudaEventDestroy(done[k]);
        }
    }
    StepMirror(const StepMirror&) = delete;
    StepMirror& operator=(const StepMirror&) = delete;
};

struct Workspace {
    int64_t n = 0;
    int m = 0;
    DevBuf<double> V, Z, w, r, ax, best, trial, tmp;
    DevBuf<double> ns1, ns2, ns_partials;   // the projected operator's scratch
    DevBuf<double> mpartial;   // (kChunk + 1) x kWideBlocks partial sums of the multi-dot
    std::unique_ptr<StepMirror> mirror;
};

Workspace& workspace(cfdxg_context* ctx, int64_t n, int m) {
    auto ws = std::static_pointer_cast<Workspace>(ctx->krylov_workspace);
    if (!ws) {
        ws = std::make_shared<Workspace>();
        ctx->krylov_workspace = ws;
    }
    if (ws->n != n || ws->m < m) {
        const int mm = std::max(m, ws->n == n ? ws->m : 0);
        ws->V.resize(static_cast<size_t>(mm + 1) * n);
        ws->Z.resize(static_cast<size_t>(mm) * n);
        ws->w.resize(n); ws->r.resize(n); ws->ax.resize(n); ws->best.resize(n);
        ws->trial.resize(n); ws->tmp.resize(n);
        ws->ns1.resize(n); ws->ns2.resize(n);
        ws->ns_partials.resize(kNsMaxBlocks);
        ws->mpartial.resize(static_cast<size_t>(kChunk + 1) * kWideBlocks);
        ws->n = n;
        ws->m = mm;
    }
    if (!ws->mirror) ws->mirror = std::make_unique<StepMirror>();
    return *ws;
}

class Engine {
public:
    Engine(cfdxg_context* ctx, const cfdxg_matrix* A) : ctx_(ctx), A_(A), n_(static_cast<int>(A->n)) {
        sc_ = ctx->scratch.scalars;
    }
    double* slot(int s) const { return sc_ + s; }
    int gb() const { return blocks_for(n_, kT); }
    int rb() const { return reduce_blocks(n_); }

    // Live profiler classes (algorithmic bytes: FP64 vectors of n, each read
    // or written once): krylov_norm, krylov_dot, gram_schmidt_dot,
    // gram_schmidt_axpy, krylov_scale, true_residual, krylov_update.
    double nb() const { return 8.0 * n_; }
    void norm2(const double* a, int out) {
        ProfScope ps(ctx_, "krylov_norm", 2.0 * nb());
        launch_pdl(ctx_->stream, k_absmax, rb(), kT, n_, a, ctx_->scratch.partial, ctx_->scratch.ticket,
                                                slot(kMax), slot(kInvalid));
        check_launch(ctx_);
        launch_pdl(ctx_->stream, k_sumsq, rb(), kT, n_, a, slot(kMax), slot(kInvalid), ctx_->scratch.partial,
                                               ctx_->scratch.ticket, slot(out));
        check_launch(ctx_);
    }
    void dot(const double* a, const double* b, int out) {
        ProfScope ps(ctx_, "krylov_dot", 2.0 * nb());
        launch_pdl(ctx_->stream, k_dot, rb(), kT, n_, a, b, ctx_->scratch.partial, ctx_->scratch.ticket, slot(out));
        check_launch(ctx_);
    }
    // w -= H[coef] v, then H[out] = u . w
    void axpy_dot(double* w, const double* v, int coef, const double* u, int out) {
        ProfScope ps(ctx_, "gram_schmidt_axpy_dot", 4.0 * nb());
        launch_pdl(ctx_->stream, k_axpy_dot, rb(), kT, n_, w, v, slot(coef), u, ctx_->scratch.partial,
                                                  ctx_->scratch.ticket, slot(out));
        check_launch(ctx_);
    }
    // w -= H[coef] v, then the norm of w into slot out (two passes, as norm2)
    void axpy_norm2(double* w, const double* v, int coef, int out) {
        ProfScope ps(ctx_, "gram_schmidt_axpy_norm", 4.0 * nb());
        launch_pdl(ctx_->stream, k_axpy_absmax, rb(), kT, n_, w, v, slot(coef), ctx_->scratch.partial,
                                                     ctx_->scratch.ticket, slot(kMax), slot(kInvalid));
        check_launch(ctx_);
        launch_pdl(ctx_->stream, k_sumsq, rb(), kT, n_, w, slot(kMax), slot(kInvalid), ctx_->scratch.partial,
                                               ctx_->scratch.ticket, slot(out));
        check_launch(ctx_);
    }
    // h[out + i] = v_i . w for i <= j (classical Gram-Schmidt), in chunks
    int wb() const { return std::min(kWideBlocks, blocks_for(n_, kT)); }
    void multidot(const double* V, int count, const double* w, int out, double* mpartial) {
        for (int i0 = 0; i0 < count; i0 += kChunk) {
            const int c = std::min(kChunk, count - i0);
            ProfScope ps(ctx_, "gram_schmidt_dot", (c + 1.0) * nb());
            launch_pdl(ctx_->stream, k_multidot, wb(), kT, n_, V, i0, c, w, mpartial, ctx_->scratch.ticket,
                                                      slot(out + i0));
            check_launch(ctx_);
        }
    }
    // w -= sum_i h[coef + i] v_i, then (last) the norm of w into slot out
    void multi_axpy(const double* V, int count, int coef, double* w, int norm_out) {
        for (int i0 = 0; i0 < count; i0 += kChunk) {
            const int c = std::min(kChunk, count - i0);
            const bool last = i0 + c == count && norm_out >= 0;
            ProfScope ps(ctx_, "gram_schmidt_axpy", (c + 2.0) * nb());
            if (last)
                launch_pdl(ctx_->stream, k_multi_axpy<true>, wb(), kT, n_, V, i0, c, slot(coef + i0), w,
                                                                 ctx_->scratch.partial, ctx_->scratch.ticket,
                                                                 slot(kMax), slot(kInvalid));
            else
                launch_pdl(ctx_->stream, k_multi_axpy<false>, blocks_for(n_, kT), kT, n_, V, i0, c, slot(coef + i0), w, nullptr,
                                                                  nullptr, nullptr, nullptr);
            check_launch(ctx_);
        }
        if (norm_out >= 0) {
            ProfScope ps(ctx_, "krylov_norm", nb());
            launch_pdl(ctx_->stream, k_sumsq, rb(), kT, n_, w, slot(kMax), slot(kInvalid), ctx_->scratch.partial,
                                                   ctx_->scratch.ticket, slot(norm_out));
            check_launch(ctx_);
        }
    }
    // Two passes of classical Gram-Schmidt of w against v_0..v_{count-1}
    // (count <= kChunk) in three passes over the basis: h1 = V^T w (with the
    // action norm), w -= V h1 fused with h2 = V^T w, w -= V h2 fused with
    // ||w||.  Fills slots kH1.., kH2.., kAction and kHnext.
    // One resident wave of each pass (a fixed partition for a given count and
    // GPU, so the sums stay deterministic).
    template <auto K>
    int gs_grid() const {
        return std::min({resident_per_sm<K>() * ctx_->sm_count, kMaxReduceBlocks, blocks_for(n_, kT)});
    }
    void gram_schmidt_cgs2_fused(const double* V, int count, double* w, double* mpartial) {
        with_basis_count(count, [&](auto cc) {
            constexpr int C = decltype(cc)::value;
            {
                ProfScope ps(ctx_, "gram_schmidt_dot", (count + 1.0) * nb());
                launch_pdl(ctx_->stream, k_gs_first<C>, gs_grid<k_gs_first<C>>(), kT, n_, V, static_cast<const double*>(w), mpartial,
                           ctx_->scratch.ticket, slot(kH1));
                check_launch(ctx_);
            }
            {
                ProfScope ps(ctx_, "gram_schmidt_axpy_dot", (count + 2.0) * nb());
                launch_pdl(ctx_->stream, k_gs_axpy_dot<C>, gs_grid<k_gs_axpy_dot<C>>(), kT, n_, V, static_cast<const double*>(slot(kH1)),
                           w, mpartial, ctx_->scratch.ticket, slot(kH2));
                check_launch(ctx_);
            }
            {
                ProfScope ps(ctx_, "gram_schmidt_axpy_norm", (count + 2.0) * nb());
                launch_pdl(ctx_->stream, k_gs_axpy_norm<C>, gs_grid<k_gs_axpy_norm<C>>(), kT, n_, V, static_cast<const double*>(slot(kH2)),
                           w, ctx_->scratch.partial, ctx_->scratch.ticket, slot(kHnext));
                check_launch(ctx_);
            }
        });
    }
    void sqrt_slot(int from, int to) {
        k_sqrt_slot<<<1, 1, 0, ctx_->stream>>>(slot(from), slot(to));
        check_launch(ctx_);
    }
    void axpy_neg(double* w, const double* v, int coef) {
        ProfScope ps(ctx_, "gram_schmidt_axpy", 3.0 * nb());
        launch_pdl(ctx_->stream, k_axpy_neg, gb(), kT, n_, w, v, slot(coef));
        check_launch(ctx_);
    }
    void div(const double* w, int d, double* v) {
        ProfScope ps(ctx_, "krylov_scale", 2.0 * nb());
        launch_pdl(ctx_->stream, k_div, gb(), kT, n_, w, slot(d), v);
        check_launch(ctx_);
    }
    void residual(const double* b, const double* x, double* r) {
        ProfScope ps(ctx_, "true_residual", 12.0 * A_->nnz + 4.0 * (n_ + 1) + 3.0 * nb());
        launch_pdl(ctx_->stream, k_true_residual, gb(), kT, n_, A_->ro.get(), A_->co.get(), A_->va.get(), b, x, r);
        check_launch(ctx_);
    }
    void spmv(const double* x, double* y) { spmv_fp64(ctx_, A_, x, y); }
    // Projection onto the complement of the constant null space,
    // v -= (v . e) e (null_space.h:64-71), the sum in a fixed order.
    void set_projection(double e, Workspace& ws) {
        ns_e_ = e;
        ns1_ = ws.ns1.get();
        ns2_ = ws.ns2.get();
        nsp_ = ws.ns_partials.get();
    }
    bool projected() const { return ns_e_ != 0.0; }
    double projection_entry() const { return ns_e_; }
    void project(double* v) {
        ProfScope ps(ctx_, "null_space_projection", 3.0 * nb());
        enqueue_remove_constant<double>(ctx_->stream, n_, v, nsp_, false, false, ns_e_);
        check_launch(ctx_);
        count_launch(ctx_);
    }
    // The Krylov operator: A, or P A P under a projected null space
    // (projected_gmres.h:122-131).
    void op(const double* x, double* y) {
        if (!projected()) {
            spmv(x, y);
            return;
        }
        copy(ns1_, x);
        project(ns1_);
        spmv(ns1_, y);
        project(y);
    }
    // r = b - op(x): the residual the Krylov solve certifies against
    void op_residual(const double* b, const double* x, double* r) {
        if (!projected()) {
            residual(b, x, r);
            return;
        }
        op(x, ns2_);
        k_sub<<<gb(), kT, 0, ctx_->stream>>>(n_, b, ns2_, r);
        check_launch(ctx_);
    }
    // z = P M P v, the ProjectedPreconditioner (projected_gmres.h:32-44); M is
    // pc, or the identity without one
    bool precondition(const RightPreconditioner* pc, const double* v, double* z, int j) {
        if (!projected()) {
            if (pc) return (*pc)(v, z, j);
            copy(z, v);
            return true;
        }
        copy(ns1_, v);
        project(ns1_);
        if (pc) {
            if (!(*pc)(ns1_, z, j)) return false;
        } else {
            copy(z, ns1_);
        }
        project(z);
        return true;
    }
    // scaled two-pass norm of count entries of a (count may exceed n)
    void norm2_n(const double* a, int count, int out) {
        const int b = reduce_blocks(count);
        launch_pdl(ctx_->stream, k_absmax, b, kT, count, a, ctx_->scratch.partial, ctx_->scratch.ticket,
                   slot(kMax), slot(kInvalid));
        check_launch(ctx_);
        launch_pdl(ctx_->stream, k_sumsq, b, kT, count, a, slot(kMax), slot(kInvalid), ctx_->scratch.partial,
                   ctx_->scratch.ticket, slot(out));
        check_launch(ctx_);
    }
    void copy(double* dst, const double* src) {
        CFDXG_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * n_, cudaMemcpyDeviceToDevice, ctx_->stream));
    }
    void update(const double* x, const double* Z, const std::vector<double>& y, int used, double* out) {
        if (used > 0)
            CFDXG_CUDA(cudaMemcpyAsync(slot(kY), y.data(), sizeof(double) * used, cudaMemcpyHostToDevice,
                                       ctx_->stream));
        ProfScope ps(ctx_, "krylov_update", (used + 2.0) * nb());
        launch_pdl(ctx_->stream, k_update, gb(), kT, n_, x, Z, slot(kY), used, out);
        check_launch(ctx_);
    }
    void neg(const double* a, double* b) {
        k_neg<<<gb(), kT, 0, ctx_->stream>>>(n_, a, b);
        check_launch(ctx_);
    }
    void add(double* x, const double* y) {
        k_add<<<gb(), kT, 0, ctx_->stream>>>(n_, x, y);
        check_launch(ctx_);
    }
    // Copies slots [0, count) to the host and synchronises; returns the status word.
    int fetch(int count) {
        CFDXG_CUDA(cudaMemcpyAsync(ctx_->scratch.host_scalars, sc_, sizeof(double) * count,
                                   cudaMemcpyDeviceToHost, ctx_->stream));
        return read_status(ctx_);
    }
    double host(int s) const { return ctx_->scratch.host_scalars[s]; }
    // Queues the copy of slots [0, count) and of the status word into mirror
    // buffer k, then marks it with the buffer's event (no synchronisation).
    void fetch_async(StepMirror& M, int k, int count) {
        CFDXG_CUDA(cudaMemcpyAsync(M.scalars[k], sc_, sizeof(double) * count, cudaMemcpyDeviceToHost,
                                   ctx_->stream));
        CFDXG_CUDA(cudaMemcpyAsync(M.status[k], ctx_->scratch.status, sizeof(int), cudaMemcpyDeviceToHost,
                                   ctx_->stream));
        CFDXG_CUDA(cudaEventRecord(M.done[k], ctx_->stream));
    }
    double scalar(int s) {   // read one slot
        fetch(s + 1);
        return host(s);
    }

private:
    cfdxg_context* ctx_;
    const cfdxg_matrix* A_;
    int n_;
    double* sc_;
    double ns_e_ = 0.0;
    double *ns1_ = nullptr, *ns2_ = nullptr, *nsp_ = nullptr;
};

// ---------------------------------------------------------------- CG kernels
// CG scalar slots (below GMRES's Hessenberg area)
enum CgSlot : int {
    kCgPAp = 8, kCgRsOld = 9, kCgRsNew = 10, kCgZBad = 11, kCgRes = 12, kCgRR2 = 13, kCgXBad = 14,
    kCgMax = 15, kCgInvalid = 16, kCgCount = 17
};

// out_dot = sum_i r_i z_i (the k_dot partition and order); out_bad = 1 when a
// z_i is not finite (cg_solver.h:213-215, the preconditioner's result check).
__global__ void k_dot_check(int n, const double* __restrict__ r, const double* __restrict__ z, double* partial,
                            unsigned* ticket, double* out_dot, double* out_bad) {
    __shared__ double sm[32];
    double s = 0.0, bad = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double zi = z[i];
        if (!isfinite(zi)) bad = 1.0;
        s += r[i] * zi;
    }
    s = block_sum(s, sm);
    bad = block_max(bad, sm);
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = s; partial[2 * blockIdx.x + 1] = bad; }
    if (last_block(ticket)) {
        double t = 0.0, bb = 0.0;
        for (int q = threadIdx.x; q < gridDim.x; q += blockDim.x) {
            t += partial[2 * q];
            bb = fmax(bb, partial[2 * q + 1]);
        }
        t = block_sum(t, sm);
        bb = block_max(bb, sm);
        if (threadIdx.x == 0) { *out_dot = t; *out_bad = bb; *ticket = 0; }
    }
}

// x += alpha p, r -= alpha Ap with alpha = rsold / pAp, only when p^T A p > 0
// and alpha are finite (cg_solver.h:287-313); bad = 1 on a non-finite x_i or r_i.
__global__ void k_cg_update(int n, double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                            const double* __restrict__ Ap, double* slots) {
    const double pAp = slots[kCgPAp];
    if (!(pAp > 0.0) || !isfinite(pAp)) return;
    const double alpha = slots[kCgRsOld] / pAp;
    if (!isfinite(alpha)) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double xi = x[i] + alpha * p[i];
    const double ri = r[i] - alpha * Ap[i];
    x[i] = xi;
    r[i] = ri;
    if (!isfinite(xi) || !isfinite(ri)) slots[kCgXBad] = 1.0;
}

// p = z + beta p with beta = rsnew / rsold (cg_solver.h:532-539)
__global__ void k_cg_direction(int n, double* __restrict__ p, const double* __restrict__ z, const double* slots) {
    const double beta = slots[kCgRsNew] / slots[kCgRsOld];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = z[i] + beta * p[i];
}

// flag = 1 when any of a[0..n) is not finite
__global__ void k_any_nonfinite(int64_t n, const double* __restrict__ a, double* flag) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        if (!isfinite(a[i])) *flag = 1.0;
}

// krylov_controls.h:28-51
int choose_restart(int current, double reduction, const KrylovControls& c) {
    if (!c.adaptive_restart) return std::clamp(current, c.restart_min, c.restart_max);
    if (reduction > c.target_reduction_per_cycle * 2.0)
        return current > c.restart_max - 5 ? c.restart_max : current + 5;
    if (reduction < c.target_reduction_per_cycle * 0.5) return std::max(c.restart_min, current - 5);
    return std::clamp(current, c.restart_min, c.restart_max);
}

}  // namespace

KrylovResult gmres_solve(cfdxg_context* ctx, const cfdxg_matrix* A, const double* b, double* x,
                         int restart, int64_t max_iter, double tolerance, const RightPreconditioner* pc,
                         const KrylovControls& controls, const IterationObserver* observer, double projection) {
    KrylovResult result;
    const int64_t n = A->n;
    if (n == 0 || restart <= 0 || max_iter == 0 || !std::isfinite(tolerance) || tolerance <= 0.0) {
        result.status = CFDXG_NOT_APPLICABLE;
        return result;
    }
    if (controls.restart_min <= 0 || controls.restart_max < controls.restart_min ||
        !std::isfinite(controls.target_reduction_per_cycle) || controls.target_reduction_per_cycle <= 0.0 ||
        controls.target_reduction_per_cycle >= 1.0 || !std::isfinite(controls.residual_replacement_gap_ratio) ||
        controls.residual_replacement_gap_ratio < 1.0) {
        result.status = CFDXG_NOT_APPLICABLE;
        return result;
    }
    if (n > std::numeric_limits<int>::max()) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "system too large");
    Engine E(ctx, A);
    clear_status(ctx);
    int current_restart = std::clamp(restart, controls.restart_min, controls.restart_max);
    if (n < current_restart) current_restart = static_cast<int>(n);
    if (projection != 0.0) E.set_projection(projection, workspace(ctx, n, current_restart));

    E.norm2(b, kNorm);
    const double b_norm = E.scalar(kNorm);
    if (!std::isfinite(b_norm)) {
        result.status = CFDXG_DIVERGED;
        return result;
    }
    if (b_norm == 0.0) {
        // gmres_solver.h:64-134: b == 0 with x0 != 0 -> solve A y = -A x0, certify on ||A x0||.
        Workspace& ws = workspace(ctx, n, current_restart);
        E.op(x, ws.ax.get());
        E.norm2(ws.ax.get(), kNorm);
        const double ax0_norm = E.scalar(kNorm);
        if (!std::isfinite(ax0_norm)) {
            result.status = CFDXG_DIVERGED;
            result.residual = ax0_norm;
            result.residual_relative = ax0_norm;
            return result;
        }
        if (ax0_norm > 0.0) {
            DevBuf<double> shifted(n), y(n);
            E.neg(ws.ax.get(), shifted.get());
            y.zero(ctx->stream);
            const KrylovResult sh = gmres_solve(ctx, A, shifted.get(), y.get(), restart, max_iter, tolerance, pc,
                                                controls, observer, projection);
            Workspace& ws2 = workspace(ctx, n, current_restart);
            E.add(x, y.get());
            E.op_residual(b, x, ws2.r.get());
            E.norm2(ws2.r.get(), kNorm);
            const double residual = E.scalar(kNorm);
            const double relative = residual / ax0_norm;
            const bool certified = std::isfinite(residual) && std::isfinite(relative) && relative <= tolerance;
            result = sh;
            result.status = certified ? CFDXG_CONVERGED
                                      : (sh.status == CFDXG_NOT_APPLICABLE ? CFDXG_NOT_APPLICABLE : CFDXG_DIVERGED);
            result.residual = residual;
            result.residual_relative = relative;
            return result;
        }
    }
    const double rhs_scale = std::max(b_norm, 1e-300);
    const double tol = b_norm == 0.0 ? 0.0 : tolerance * b_norm;

    Workspace* ws = &workspace(ctx, n, current_restart);
    auto true_residual = [&]() {
        E.op_residual(b, x, ws->r.get());
        E.norm2(ws->r.get(), kBeta);
        return E.scalar(kBeta);
    };

    double beta = true_residual();
    if (!std::isfinite(beta)) {
        result.status = CFDXG_DIVERGED;
        result.residual = beta;
        return result;
    }
    if (b_norm == 0.0) {
        E.norm2(x, kNorm);
        const double x_norm = E.scalar(kNorm);
        const double ref_scale = std::max({x_norm, 1.0, 1e-300});
        const double tol_b0 = tolerance * ref_scale;
        result.status = beta <= tol_b0 ? CFDXG_CONVERGED : CFDXG_DIVERGED;
        result.iterations = 0;
        result.residual = beta;
        result.residual_relative = beta / ref_scale;
        return result;
    }
    if (beta <= tol) {
        result.status = CFDXG_CONVERGED;
        result.iterations = 0;
        result.residual = beta;
        result.residual_relative = beta / rhs_scale;
        return result;
    }

    int64_t iterations = 0;
    double previous_cycle_residual = beta;
    E.copy(ws->best.get(), x);
    double best_residual = beta;
    auto restore_best = [&]() { E.copy(x, ws->best.get()); };
    auto fail = [&](int status) {
        restore_best();
        result.status = status;
        result.iterations = iterations;
        result.residual = best_residual;
        result.residual_relative = best_residual / rhs_scale;
        CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
        return result;
    };

    std::vector<double> h, cs, sn, g, y;
    while (iterations < max_iter) {
        ws = &workspace(ctx, n, current_restart);
        const int m = current_restart;
        h.assign(static_cast<size_t>(m + 1) * m, 0.0);
        cs.assign(m, 0.0);
        sn.assign(m, 0.0);
        g.assign(m + 1, 0.0);
        y.assign(m, 0.0);
        auto H = [&](int i, int j) -> double& { return h[static_cast<size_t>(i) * m + j]; };
        double* V = ws->V.get();
        double* Z = ws->Z.get();
        auto v = [&](int j) { return V + static_cast<size_t>(j) * n; };
        auto z = [&](int j) { return Z + static_cast<size_t>(j) * n; };

        beta = true_residual();
        if (!std::isfinite(beta)) return fail(CFDXG_DIVERGED);
        if (beta <= tol) break;
        E.div(ws->r.get(), kBeta, v(0));
        g[0] = beta;

        int used = 0;
        double estimated_residual = beta;
        bool arnoldi_breakdown = false;
        bool reliable_restart = false;

        // One Arnoldi step on the device: z_j = M^-1 v_j, w = A z_j, the
        // Gram-Schmidt passes into the H slots, v_{j+1} = w / h_{j+1,j}, and
        // the queued copy of the step's slots into mirror buffer j & 1.
        StepMirror& mirror = *ws->mirror;
        auto enqueue_step = [&](int jj) -> bool {
            if (!E.precondition(pc, v(jj), z(jj), jj)) return false;
            E.op(z(jj), ws->w.get());
            double* w = ws->w.get();
            if (controls.classical_gram_schmidt && jj + 1 <= kChunk) {
                // classical Gram-Schmidt twice in three fused passes; the
                // action norm comes from the first (slot kH1 + jj + 1)
                E.gram_schmidt_cgs2_fused(V, jj + 1, w, ws->mpartial.get());
                E.sqrt_slot(kH1 + jj + 1, kAction);
            } else if (controls.classical_gram_schmidt) {
                // two passes of classical Gram-Schmidt: h = V^T w; w -= V h, twice
                E.norm2(w, kAction);
                E.multidot(V, jj + 1, w, kH1, ws->mpartial.get());
                E.multi_axpy(V, jj + 1, kH1, w, -1);
                E.multidot(V, jj + 1, w, kH2, ws->mpartial.get());
                E.multi_axpy(V, jj + 1, kH2, w, kHnext);
            } else {
                // two passes of modified Gram-Schmidt (h = v_i . w; w -= h v_i
                // for i = 0..jj, twice), each update fused with the next dot
                E.norm2(w, kAction);
                E.dot(v(0), w, kH1);
                for (int i = 0; i < jj; ++i) E.axpy_dot(w, v(i), kH1 + i, v(i + 1), kH1 + i + 1);
                E.axpy_dot(w, v(jj), kH1 + jj, v(0), kH2);
                for (int i = 0; i < jj; ++i) E.axpy_dot(w, v(i), kH2 + i, v(i + 1), kH2 + i + 1);
                E.axpy_norm2(w, v(jj), kH2 + jj, kHnext);
            }
            E.div(w, kHnext, v(jj + 1));
            E.fetch_async(mirror, jj & 1, kH2 + jj + 1);
            return true;
        };
        // Run-ahead: step j + 1 is queued before step j's results are read
        // whenever step j is predicted not to stop the cycle (its residual
        // estimate, extrapolated from the last two, stays above 4 x tol), so
        // the GPU is not idle while the host runs the Givens update.  A step
        // queued in vain only writes z, w and v beyond the cycle's used
        // columns and H slots already copied; its results are ignored.
        double est_prev = beta, ratio_prev = 1.0;
        bool queued = enqueue_step(0);
        if (!queued) return fail(CFDXG_NOT_APPLICABLE);
        for (int j = 0; j < m && iterations < max_iter; ++j) {
            bool ahead = false, ahead_failed = false;
            if (j + 1 < m && iterations + 1 < max_iter && est_prev * ratio_prev > 4.0 * tol) {
                ahead = true;
                ahead_failed = !enqueue_step(j + 1);
            }
            CFDXG_CUDA(cudaEventSynchronize(mirror.done[j & 1]));
            const double* hs = mirror.scalars[j & 1];
            const bool preconditioned = pc || E.projected();
            if (preconditioned) ++result.preconditioner_applications;
            if (*mirror.status[j & 1] & kStatusNonFinite) {
                if (preconditioned) return fail(CFDXG_NOT_APPLICABLE);   // preconditioner produced a non-finite z
            }
            const double arnoldi_action_norm = hs[kAction];
            if (!std::isfinite(arnoldi_action_norm)) return fail(CFDXG_DIVERGED);
            for (int i = 0; i <= j; ++i) {
                H(i, j) = hs[kH1 + i];
                H(i, j) += hs[kH2 + i];
            }
            const double hnext = hs[kHnext];
            if (!std::isfinite(hnext)) return fail(CFDXG_DIVERGED);
            H(j + 1, j) = hnext;
            const double floor = 4096.0 * kEps * std::max(arnoldi_action_norm, 1e-300);
            const bool breakdown_detected = hnext <= floor && arnoldi_action_norm > 0.0;

            for (int i = 0; i < j; ++i) {
                const double h0 = H(i, j), h1 = H(i + 1, j);
                H(i, j) = cs[i] * h0 + sn[i] * h1;
                H(i + 1, j) = -sn[i] * h0 + cs[i] * h1;
            }
            const double a = H(j, j), b2 = H(j + 1, j);
            const double rho = std::hypot(a, b2);
            if (rho > 0.0) {
                cs[j] = a / rho;
                sn[j] = b2 / rho;
                H(j, j) = rho;
                H(j + 1, j) = 0.0;
                const double gj = g[j], gj1 = g[j + 1];
                g[j] = cs[j] * gj + sn[j] * gj1;
                g[j + 1] = -sn[j] * gj + cs[j] * gj1;
            }
            ++iterations;
            ++used;
            estimated_residual = std::abs(g[j + 1]);
            if (observer) (*observer)(estimated_residual);
            if (breakdown_detected) {
                arnoldi_breakdown = true;
                break;
            }
            if (estimated_residual <= tol) break;
            if (controls.residual_replacement && controls.residual_replacement_period > 0 &&
                iterations % controls.residual_replacement_period == 0) {
                std::vector<double> coef(used, 0.0);
                bool usable = true;
                for (int i = used; i-- > 0;) {
                    double sum = g[i];
                    for (int k = i + 1; k < used; ++k) sum -= H(i, k) * coef[k];
                    const double diagonal = H(i, i);
                    if (!std::isfinite(sum) || !std::isfinite(diagonal) ||
                        std::abs(diagonal) <= 128.0 * kEps * std::max(arnoldi_action_norm, 1e-300)) {
                        usable = false;
                        break;
                    }
                    coef[i] = sum / diagonal;
                }
                if (usable) {
                    E.update(x, Z, coef, used, ws->trial.get());
                    E.op_residual(b, ws->trial.get(), ws->tmp.get());
                    E.norm2(ws->tmp.get(), kNorm);
                    const double verified = E.scalar(kNorm);
                    if (std::isfinite(verified)) {
                        result.max_true_residual = std::max(result.max_true_residual, verified);
                        result.min_true_residual = std::min(result.min_true_residual, verified);
                        const double ratio = verified / std::max(estimated_residual, 1e-300);
                        result.max_true_recursive_ratio = std::max(result.max_true_recursive_ratio, ratio);
                        result.min_true_recursive_ratio = std::min(result.min_true_recursive_ratio, ratio);
                        result.max_true_recursive_gap =
                            std::max(result.max_true_recursive_gap, std::abs(verified - estimated_residual));
                        if (ratio > controls.residual_replacement_gap_ratio) {
                            reliable_restart = true;
                            break;
                        }
                    } else {
                        reliable_restart = true;
                        break;
                    }
                }
            }
            if (estimated_residual > 0.0 && est_prev > 0.0) ratio_prev = std::min(1.0, estimated_residual / est_prev);
            est_prev = estimated_residual;
            if (j + 1 < m && iterations < max_iter) {
                if (ahead ? ahead_failed : !enqueue_step(j + 1)) return fail(CFDXG_NOT_APPLICABLE);
            }
        }
        if (used == 0) break;

        std::fill(y.begin(), y.end(), 0.0);
        for (int i = used; i-- > 0;) {
            double sum = g[i];
            for (int j = i + 1; j < used; ++j) sum -= H(i, j) * y[j];
            const double diag = H(i, i);
            double h_scale = std::abs(diag);
            for (int k = 0; k < used; ++k) h_scale = std::max(h_scale, std::abs(H(k, i)));
            const double diag_floor = 128.0 * kEps * std::max(h_scale, 1e-300);
            if (std::abs(diag) <= diag_floor) {
                if (std::abs(sum) <= diag_floor) {
                    y[i] = 0.0;
                    continue;
                }
                double breakdown_residual = true_residual();
                if (!std::isfinite(breakdown_residual) || best_residual < breakdown_residual) {
                    restore_best();
                    breakdown_residual = best_residual;
                }
                result.status = CFDXG_DIVERGED;
                result.iterations = iterations;
                result.residual = breakdown_residual;
                result.residual_relative = breakdown_residual / rhs_scale;
                CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
                return result;
            }
            y[i] = sum / diag;
        }
        E.update(x, Z, y, used, x);

        beta = true_residual();
        if (reliable_restart && std::isfinite(beta)) {
            ++result.residual_replacements;
            if (result.first_residual_replacement == 0) result.first_residual_replacement = iterations;
            result.last_residual_replacement = iterations;
            const double ratio = beta / std::max(estimated_residual, 1e-300);
            result.min_true_recursive_ratio = std::min(result.min_true_recursive_ratio, ratio);
            result.max_true_recursive_ratio = std::max(result.max_true_recursive_ratio, ratio);
            result.max_true_recursive_gap = std::max(result.max_true_recursive_gap, std::abs(beta - estimated_residual));
            result.min_true_residual = std::min(result.min_true_residual, beta);
            result.max_true_residual = std::max(result.max_true_residual, beta);
        }
        if (!std::isfinite(beta)) return fail(CFDXG_DIVERGED);
        if (beta < best_residual) {
            best_residual = beta;
            E.copy(ws->best.get(), x);
        }
        if (beta <= tol) {
            result.status = CFDXG_CONVERGED;
            result.iterations = iterations;
            result.residual = beta;
            result.residual_relative = beta / rhs_scale;
            CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
            return result;
        }
        if (arnoldi_breakdown) {
            if (best_residual < beta) {
                restore_best();
                beta = best_residual;
            }
            result.status = CFDXG_DIVERGED;
            result.iterations = iterations;
            result.residual = beta;
            result.residual_relative = beta / rhs_scale;
            CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
            return result;
        }
        const double reduction = beta / std::max(previous_cycle_residual, 1e-300);
        if (!std::isfinite(reduction)) return fail(CFDXG_DIVERGED);
        if (controls.adaptive_restart) {
            current_restart = choose_restart(current_restart, reduction, controls);
            if (n < current_restart) current_restart = static_cast<int>(n);
        }
        previous_cycle_residual = beta;
    }
    if (best_residual < beta) {
        restore_best();
        beta = best_residual;
    }
    result.status = CFDXG_MAX_ITER_REACHED;
    result.iterations = iterations;
    result.residual = beta;
    result.residual_relative = beta / rhs_scale;
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    return result;
}

// ---------------------------------------------------------------- null space
double constant_null_space_entry(int64_t n) {
    // null_space.h:58-62: the ones vector over its hypot-accumulated norm
    // (:141-146), computed once per size
    static std::mutex mu;
    static int64_t last_n = -1;
    static double last_e = 0.0;
    std::lock_guard<std::mutex> lock(mu);
    if (n != last_n) {
        double norm = 0.0;
        for (int64_t i = 0; i < n; ++i) norm = std::hypot(norm, 1.0);
        last_e = 1.0 * (1.0 / norm);
        last_n = n;
    }
    return last_e;
}

NullSpaceChecks null_space_checks(cfdxg_context* ctx, const cfdxg_matrix* A, const double* b) {
    NullSpaceChecks c;
    const int64_t n = A->n;
    if (n <= 0) return c;
    if (A->nnz > std::numeric_limits<int>::max()) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "system too large");
    const double e = constant_null_space_entry(n);
    Engine E(ctx, A);
    Workspace& ws = workspace(ctx, n, 1);
    const int ni = static_cast<int>(n);
    // null_space.h:90-105 is_compatible: |b . e| <= 1e-14 + 1e-12 ||b||
    const int nb = ns_blocks(n);
    k_ns_partials<double><<<nb, kNsThreads, 0, ctx->stream>>>(ni, b, e, ws.ns_partials.get());
    check_launch(ctx);
    std::vector<double> part(ws.ns_partials.size());
    ws.ns_partials.download(part.data(), ctx->stream);
    E.norm2(b, kNorm);
    const double b_norm = E.scalar(kNorm);
    double coefficient = 0.0;
    for (int q = 0; q < nb; ++q) coefficient += part[q];
    c.component = std::sqrt(std::max(0.0, coefficient * coefficient));
    c.compatible = c.component <= 1e-14 + 1e-12 * b_norm;
    // :107-134 operator_residual: ||A e|| / ||A||_F <= 1e-12
    E.norm2_n(A->va.get(), static_cast<int>(A->nnz), kNorm);
    const double frobenius = E.scalar(kNorm);
    k_fill<<<blocks_for(n, kT), kT, 0, ctx->stream>>>(ni, e, ws.ns1.get());
    check_launch(ctx);
    E.spmv(ws.ns1.get(), ws.ns2.get());
    E.norm2(ws.ns2.get(), kNorm);
    const double product = E.scalar(kNorm);
    if (!std::isfinite(frobenius)) return c;
    c.operator_residual = product / std::max(frobenius, std::numeric_limits<double>::min());
    c.null_space = c.operator_residual <= 1e-12;
    // projected_gmres.h:53-82 is_bilateral_null_space: and ||A^T e|| <= 1e-12 ||A||_F
    ws.ns2.zero(ctx->stream);
    k_transpose_apply<<<blocks_for(n, kT), kT, 0, ctx->stream>>>(ni, A->ro.get(), A->co.get(), A->va.get(),
                                                                ws.ns1.get(), ws.ns2.get());
    check_launch(ctx);
    E.norm2(ws.ns2.get(), kNorm);
    const double transpose = E.scalar(kNorm);
    c.bilateral = c.null_space &&
                  !(transpose > 1e-12 * std::max(frobenius, std::numeric_limits<double>::min()));
    return c;
}

// projected_gmres.h:84-150 solve_projected_gmres: parameter and null-space
// checks (NOT_APPLICABLE, x untouched), a gauge-free copy of the iterate, the
// early exit when it already satisfies b in physical coordinates, the
// preconditioner setup, then FGMRES on P A P preconditioned by P M P and the
// projected result.
KrylovResult projected_gmres_solve(cfdxg_context* ctx, const cfdxg_matrix* A, const double* b, double* x,
                                   int restart, int64_t max_iter, double tolerance, const RightPreconditioner* pc,
                                   const KrylovControls& controls, const IterationObserver* observer,
                                   const std::function<bool()>* setup) {
    KrylovResult result;   // NOT_APPLICABLE
    const int64_t n = A->n;
    if (n == 0 || restart <= 0 || max_iter == 0 || !(tolerance > 0.0) || !std::isfinite(tolerance)) return result;
    if (n > std::numeric_limits<int>::max()) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "system too large");
    Engine E(ctx, A);
    Workspace& ws = workspace(ctx, n, 1);
    CFDXG_CUDA(cudaMemsetAsync(E.slot(kDot), 0, sizeof(double), ctx->stream));
    k_any_nonfinite<<<blocks_for(n, kT), kT, 0, ctx->stream>>>(n, b, E.slot(kDot));
    k_any_nonfinite<<<blocks_for(n, kT), kT, 0, ctx->stream>>>(n, x, E.slot(kDot));
    check_launch(ctx);
    if (E.scalar(kDot) > 0.0) return result;
    const NullSpaceChecks checks = null_space_checks(ctx, A, b);
    if (!checks.compatible || !checks.bilateral) return result;
    const double e = constant_null_space_entry(n);
    E.set_projection(e, ws);
    DevBuf<double> gauge_free(n);
    E.copy(gauge_free.get(), x);
    E.project(gauge_free.get());
    E.residual(b, gauge_free.get(), ws.tmp.get());
    E.norm2(ws.tmp.get(), kNorm);
    const double r0 = E.scalar(kNorm);
    E.norm2(b, kNorm);
    const double b_norm = E.scalar(kNorm);
    if (r0 == 0.0 || (b_norm > 0.0 && r0 <= tolerance * b_norm)) {
        result.status = CFDXG_CONVERGED;
        result.residual = r0;
        result.residual_relative = b_norm > 0.0 ? r0 / b_norm : 0.0;
        E.copy(x, gauge_free.get());
        CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
        return result;
    }
    if (setup && !(*setup)()) return result;
    result = gmres_solve(ctx, A, b, gauge_free.get(), restart, max_iter, tolerance, pc, controls, observer, e);
    if (result.status != CFDXG_NOT_APPLICABLE) {
        CFDXG_CUDA(cudaMemsetAsync(E.slot(kDot), 0, sizeof(double), ctx->stream));
        k_any_nonfinite<<<blocks_for(n, kT), kT, 0, ctx->stream>>>(n, gauge_free.get(), E.slot(kDot));
        check_launch(ctx);
        if (!(E.scalar(kDot) > 0.0)) {
            E.project(gauge_free.get());
            E.copy(x, gauge_free.get());
        }
    }
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    return result;
}

// ---------------------------------------------------------------- CG
// cg_solver.h:45-560 solve_cg_impl (FP64 operator and reductions, adaptive
// residual replacement, optionally the constant null space) with a
// preconditioner object.  Each
// iteration is one stream of kernels -- A p, p^T A p, the fused x/r update,
// z = M^-1 r, r^T z with the z check, the FP64 true residual b - A x and its
// scaled norm, ||r||^2 -- and one read-back of eight scalars, after which the
// host takes the reference's decisions in the reference's order.
KrylovResult cg_solve(cfdxg_context* ctx, const cfdxg_matrix* A, const double* b, double* x, int64_t max_iter,
                      double tolerance, const RightPreconditioner& pc, const std::function<bool()>* setup,
                      bool own_diagonal, bool null_space) {
    KrylovResult result;
    const int64_t n = A->n;
    if (n == 0) return result;   // NOT_APPLICABLE
    if (n > std::numeric_limits<int>::max()) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "system too large");
    if (null_space) {
        // :74-79 a compatible right-hand side and A e = 0, else NOT_APPLICABLE (x untouched)
        const NullSpaceChecks c = null_space_checks(ctx, A, b);
        if (!c.compatible || !c.null_space) return result;
    }
    Engine E(ctx, A);
    clear_status(ctx);
    const int ni = static_cast<int>(n);
    const int gb = blocks_for(n, kT);
    Workspace& ws = workspace(ctx, n, 1);
    if (null_space) E.set_projection(constant_null_space_entry(n), ws);
    auto project = [&](double* v) {
        if (null_space) E.project(v);
    };
    DevBuf<double> p(n), z(n), Ap(n);
    double* r = ws.r.get();
    double* rv = ws.tmp.get();
    auto zero_flags = [&]() {
        CFDXG_CUDA(cudaMemsetAsync(E.slot(kCgZBad), 0, sizeof(double), ctx->stream));
        CFDXG_CUDA(cudaMemsetAsync(E.slot(kCgXBad), 0, sizeof(double), ctx->stream));
    };
    auto dot_check = [&](const double* a, const double* zz, int out) {
        k_dot_check<<<E.rb(), kT, 0, ctx->stream>>>(ni, a, zz, ctx->scratch.partial, ctx->scratch.ticket,
                                                     E.slot(out), E.slot(kCgZBad));
        check_launch(ctx);
    };
    auto apply = [&]() {
        ++result.preconditioner_applications;
        if (!pc(r, z.get(), 0)) return false;
        project(z.get());                                            // :203
        return true;
    };

    // :75-85 non-finite operator, right-hand side or initial guess
    zero_flags();
    const int nnz_blocks = static_cast<int>(std::min<int64_t>(blocks_for(A->nnz, kT), 148 * 8));
    k_any_nonfinite<<<std::max(nnz_blocks, 1), kT, 0, ctx->stream>>>(A->nnz, A->va.get(), E.slot(kCgXBad));
    k_any_nonfinite<<<gb, kT, 0, ctx->stream>>>(n, b, E.slot(kCgXBad));
    k_any_nonfinite<<<gb, kT, 0, ctx->stream>>>(n, x, E.slot(kCgXBad));
    check_launch(ctx);
    if (null_space) {
        // :93 the gauge removed from the initial guess, once it is known to be finite
        E.fetch(kCgCount);
        if (E.host(kCgXBad) > 0.0) {
            result.status = CFDXG_DIVERGED;
            return result;
        }
        project(x);
    }
    // :149-169 r = b - A x before any preconditioner work
    E.residual(b, x, rv);
    project(rv);                                                     // :149
    E.norm2(b, kCgMax);                 // ||b|| (slots kMax/kInvalid are the norm's own scratch)
    E.norm2(rv, kCgRes);
    E.fetch(kCgCount);
    if (E.host(kCgXBad) > 0.0) {
        result.status = CFDXG_DIVERGED;
        return result;
    }
    const double b_norm = E.host(kCgMax);
    const double initial = E.host(kCgRes);
    const double homogeneous = b_norm == 0.0 ? initial : 0.0;
    const double reference = b_norm > 0.0 ? b_norm : initial;
    const double tol_abs = tolerance * reference;
    auto finish = [&](int status, int64_t it, double res) {
        result.status = status;
        result.iterations = it;
        result.residual = res;
        result.residual_relative = reference > 0.0 ? res / reference : 0.0;
        CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
        return result;
    };
    // :108-131 failure reports carry the recomputed FP64 residual of x
    auto failed = [&](int status, int64_t it, double res) {
        result.status = status;
        result.iterations = it;
        result.residual = res;
        result.residual_relative = b_norm > 0.0 ? res / b_norm
                                   : (homogeneous > 0.0 ? res / homogeneous
                                                        : (res == 0.0 ? 0.0 : std::numeric_limits<double>::infinity()));
        CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
        return result;
    };
    if (initial <= tol_abs) return finish(CFDXG_CONVERGED, 0, initial);
    if (setup && !(*setup)()) return failed(CFDXG_NOT_APPLICABLE, 0, initial);
    E.copy(r, rv);
    zero_flags();
    if (!apply()) return failed(CFDXG_NOT_APPLICABLE, 0, initial);
    dot_check(r, z.get(), kCgRsOld);
    E.copy(p.get(), z.get());
    E.fetch(kCgCount);
    if (E.host(kCgZBad) > 0.0) return failed(CFDXG_NOT_APPLICABLE, 0, initial);
    double rsold = E.host(kCgRsOld);
    if (!std::isfinite(rsold)) return failed(CFDXG_DIVERGED, 0, initial);
    if (!(rsold > 0.0)) return failed(CFDXG_NOT_APPLICABLE, 0, initial);

    double at_last_replacement = std::numeric_limits<double>::infinity();
    for (int64_t iter = 1; iter <= max_iter; ++iter) {
        zero_flags();
        E.spmv(p.get(), Ap.get());
        project(Ap.get());                                           // :262
        E.dot(p.get(), Ap.get(), kCgPAp);
        k_cg_update<<<gb, kT, 0, ctx->stream>>>(ni, x, r, p.get(), Ap.get(), E.slot(0));
        check_launch(ctx);
        project(x);                                                  // :295-298
        project(r);
        if (!apply()) return failed(CFDXG_NOT_APPLICABLE, iter, std::numeric_limits<double>::quiet_NaN());
        dot_check(r, z.get(), kCgRsNew);
        E.residual(b, x, rv);
        E.norm2(rv, kCgRes);
        E.dot(r, r, kCgRR2);
        E.fetch(kCgCount);
        const double pAp = E.host(kCgPAp);
        const double res = E.host(kCgRes);
        if (!(pAp > 0.0) || !std::isfinite(pAp)) return failed(CFDXG_NOT_APPLICABLE, iter, res);
        if (!std::isfinite(rsold / pAp)) return failed(CFDXG_DIVERGED, iter, res);
        if (E.host(kCgXBad) > 0.0) return failed(CFDXG_DIVERGED, iter, res);
        if (E.host(kCgZBad) > 0.0) return failed(CFDXG_NOT_APPLICABLE, iter, res);
        const double rsnew = E.host(kCgRsNew);
        if (!std::isfinite(rsnew)) return failed(CFDXG_DIVERGED, iter, res);
        if (res <= tol_abs) return finish(CFDXG_CONVERGED, iter, res);
        if (own_diagonal) {
            // :321-352 the solver's own diagonal: replace the recursive residual
            // when it claims convergence that b - A x does not confirm
            const double rr = std::sqrt(E.host(kCgRR2));
            if (std::isfinite(rr) && rr <= tol_abs && res > tol_abs) {
                ++result.residual_replacements;
                if (result.first_residual_replacement == 0) result.first_residual_replacement = iter;
                result.last_residual_replacement = iter;
                E.copy(r, rv);
                project(r);                                          // :376
                zero_flags();
                if (!apply()) return failed(CFDXG_NOT_APPLICABLE, iter, res);
                dot_check(r, z.get(), kCgRsOld);
                E.copy(p.get(), z.get());
                E.fetch(kCgCount);
                const double replaced = E.host(kCgRsOld);
                if (E.host(kCgZBad) > 0.0) return failed(CFDXG_NOT_APPLICABLE, iter, res);
                if (!std::isfinite(replaced) || !(replaced > 0.0)) return finish(CFDXG_MAX_ITER_REACHED, iter, res);
                rsold = replaced;
                continue;
            }
            k_cg_direction<<<gb, kT, 0, ctx->stream>>>(ni, p.get(), z.get(), E.slot(0));
            check_launch(ctx);
            project(p.get());                                        // :558
            CFDXG_CUDA(cudaMemcpyAsync(E.slot(kCgRsOld), E.slot(kCgRsNew), sizeof(double), cudaMemcpyDeviceToDevice,
                                       ctx->stream));
            rsold = rsnew;
            continue;
        }
        // :399-525 adaptive residual replacement and collapse repair
        const double rr = std::sqrt(E.host(kCgRR2));
        const double gap = std::abs(res - rr);
        const double scale = std::max(res, rr);
        result.max_true_recursive_gap = std::max(result.max_true_recursive_gap, gap);
        if (rr > 0.0 && std::isfinite(rr) && std::isfinite(res / rr)) {
            result.min_true_recursive_ratio = std::min(result.min_true_recursive_ratio, res / rr);
            result.max_true_recursive_ratio = std::max(result.max_true_recursive_ratio, res / rr);
        }
        result.max_true_residual = std::max(result.max_true_residual, res);
        result.min_true_residual = std::min(result.min_true_residual, res);
        const bool progress = res < 0.5 * at_last_replacement;
        const bool collapsed = !(rsnew > 0.0);
        const bool adaptive = std::isfinite(rr) && scale > 0.0 && gap > 0.25 * scale && progress;
        const bool repair = collapsed && progress;
        if (collapsed && !repair) return finish(CFDXG_MAX_ITER_REACHED, iter, res);
        if (adaptive || repair) {
            ++result.residual_replacements;
            at_last_replacement = res;
            if (result.first_residual_replacement == 0) result.first_residual_replacement = iter;
            result.last_residual_replacement = iter;
            E.copy(r, rv);
            project(r);                                              // :517
            zero_flags();
            if (!apply()) return failed(CFDXG_NOT_APPLICABLE, iter, res);
            dot_check(r, z.get(), kCgRsOld);
            E.copy(p.get(), z.get());
            E.fetch(kCgCount);
            const double replaced = E.host(kCgRsOld);
            if (E.host(kCgZBad) > 0.0 || !std::isfinite(replaced) || !(replaced > 0.0))
                return failed(CFDXG_NOT_APPLICABLE, iter, res);
            rsold = replaced;
            continue;
        }
        k_cg_direction<<<gb, kT, 0, ctx->stream>>>(ni, p.get(), z.get(), E.slot(0));
        check_launch(ctx);
        project(p.get());                                            // :558
        CFDXG_CUDA(cudaMemcpyAsync(E.slot(kCgRsOld), E.slot(kCgRsNew), sizeof(double), cudaMemcpyDeviceToDevice,
                                   ctx->stream));
        rsold = rsnew;
    }
    E.residual(b, x, rv);
    E.norm2(rv, kCgRes);
    return finish(CFDXG_MAX_ITER_REACHED, max_iter, E.scalar(kCgRes));
}

void enqueue_dot(cfdxg_context* ctx, int64_t n, const double* a, const double* b, double* out) {
    launch_pdl(ctx->stream, k_dot, reduce_blocks(n), kT, static_cast<int>(n), a, b, ctx->scratch.partial,
                                                    ctx->scratch.ticket, out);
    check_launch(ctx);
}

double device_norm2(cfdxg_context* ctx, const cfdxg_matrix* A, const double* a) {
    Engine E(ctx, A);
    E.norm2(a, kNorm);
    return E.scalar(kNorm);
}

double device_residual_norm(cfdxg_context* ctx, const cfdxg_matrix* A, const double* b, const double* x) {
    Engine E(ctx, A);
    Workspace& ws = workspace(ctx, A->n, 1);
    E.residual(b, x, ws.tmp.get());
    E.norm2(ws.tmp.get(), kNorm);
    return E.scalar(kNorm);
}

}  // namespace cfdxg
