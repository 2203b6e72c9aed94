// nullspace.cuh -- removal of a constant component on the device.
//
// Both forms are "sum, then subtract a constant":
//  * the AMG cycle's remove_constant (core/linalg/amg_preconditioner.h:1310-1319):
//    v -= (sum_i v_i) / n;
//  * the Krylov projector's remove with the normalised constant vector, every
//    entry e (core/linalg/null_space.h:64-71): v -= (sum_i v_i e) e.
// The sum runs in a fixed order -- per-block sums of contiguous chunks, the
// block sums then added in block order by every block of the second kernel --
// so a result never depends on scheduling.  With `in_order` one thread sums
// v_0, v_1, ... as the reference does, which makes the removal bit-identical
// to the reference's (used by the cycle's reference_order mode, on the small
// systems the parity tests run).
#pragma once
#include <algorithm>

#include "device.cuh"

namespace cfdxg {

constexpr int kNsThreads = 256;
constexpr int kNsMaxBlocks = 296;   // 2 x 148 SMs

inline int ns_blocks(int64_t n) {
    const int64_t b = (n + kNsThreads * 8 - 1) / (kNsThreads * 8);
    return static_cast<int>(b < 1 ? 1 : (b > kNsMaxBlocks ? kNsMaxBlocks : b));
}

// partials[block] = sum over the block's contiguous chunk of v_i * scale
template <class V>
__global__ void k_ns_partials(int n, const V* __restrict__ v, double scale, double* __restrict__ partials) {
    __shared__ double sm[32];
    const int chunk = (n + gridDim.x - 1) / gridDim.x;
    const int b = blockIdx.x * chunk;
    const int e = min(n, b + chunk);
    double s = 0.0;
    for (int i = b + threadIdx.x; i < e; i += blockDim.x) s += static_cast<double>(v[i]) * scale;
    s = block_sum(s, sm);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// partials[0] = v_0 * scale + v_1 * scale + ..., one thread, in index order
template <class V>
__global__ void k_ns_sum_in_order(int n, const V* __restrict__ v, double scale, double* __restrict__ partials) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += static_cast<double>(v[i]) * scale;
    partials[0] = s;
}

// c = total / n (mean) or total * e (projection), total = the partials in
// block order; then v_i -= c
template <class V>
__global__ void k_ns_subtract(int n, V* __restrict__ v, const double* __restrict__ partials, int nparts,
                              double e, int mean) {
    __shared__ double c_s;
    if (threadIdx.x < 32) {
        double t;
        if (nparts == 1) {
            t = partials[0];
        } else {
            t = 0.0;
            for (int q = threadIdx.x; q < nparts; q += 32) t += partials[q];
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        }
        if (threadIdx.x == 0) c_s = mean ? t / static_cast<double>(n) : t * e;
    }
    __syncthreads();
    const double c = c_s;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        v[i] = static_cast<V>(static_cast<double>(v[i]) - c);
}

// Enqueues the removal on `stream`: mean subtraction (mean = true) or the
// projection with entry e.  partials holds at least kNsMaxBlocks values.
template <class V>
void enqueue_remove_constant(cudaStream_t stream, int n, V* v, double* partials, bool in_order, bool mean,
                             double e) {
    if (n <= 0) return;
    const int nb = in_order ? 1 : ns_blocks(n);
    if (in_order) k_ns_sum_in_order<V><<<1, 32, 0, stream>>>(n, v, mean ? 1.0 : e, partials);
    else k_ns_partials<V><<<nb, kNsThreads, 0, stream>>>(n, v, mean ? 1.0 : e, partials);
    const int sb = std::min(blocks_for(n, kNsThreads), 4 * 148);
    k_ns_subtract<V><<<sb, kNsThreads, 0, stream>>>(n, v, partials, nb, e, mean ? 1 : 0);
}

}  // namespace cfdxg
