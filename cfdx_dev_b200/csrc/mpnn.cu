// mpnn.cu -- learned message-passing preconditioner on the matrix graph.
//
// Network (no counterpart in the reference; the FP64 oracle is
// oracle/mpnn_oracle.py, whose parameter layout this file shares):
//   s = rms(r);  x_i = [r_i/s, f_V, f_P, f_D]   (standardised log volume, log a_P, log a_ii)
//   h = relu(W_in x + b_in)
//   4 rounds:  a_i = sum_j w_ij h_j  (w_ij = -a_ij / sqrt(a_ii a_jj));
//              h_i += W2 relu(W1 [h_i, a_i] + b1) + b2
//   N(r)_i = s (w_out . h_i + b_out) / a_ii
//
// Training kernels run in FP32 (forward, backward, Adam) with deterministic
// weight-gradient reductions: each warp owns a fixed set of cells, warps are
// combined in a fixed order per block and blocks in a fixed order at the end.
// Inference runs each round as one fused kernel: the neighbour gather builds
// [h, a] in shared memory as BF16 and both MLP layers run on the tensor cores
// (mma.sync m16n8k16, BF16 operands, FP32 accumulation); the state h is
// stored as BF16 between rounds and carried in FP32 within one.
// The encoder is folded into the first round (h0 formed from r where it is
// read) and the readout into the last, so inference is four kernels.
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <random>
#include <thread>

#include "io.h"
#include "krylov.h"
#include "mpnn.h"

namespace cfdxg {
namespace mp {

constexpr int F = 32;
constexpr int R = 4;
constexpr int OFF_WIN = 0, OFF_BIN = 128;
constexpr int ROUND0 = 160, ROUND_SIZE = 3136;   // W1 2048, b1 32, W2 1024, b2 32
constexpr int OFF_W1 = 0, OFF_B1 = 2048, OFF_W2 = 2080, OFF_B2 = 3104;
constexpr int OFF_WOUT = ROUND0 + R * ROUND_SIZE;   // 12704
constexpr int OFF_BOUT = OFF_WOUT + F;              // 12736
constexpr int NP = OFF_BOUT + 1;                    // 12737
constexpr int kGridBlocks = 296;                    // fixed partition of cells for reductions
constexpr int kThreads = 128;
constexpr int kWarps = kThreads / 32;

}  // namespace mp
}  // namespace cfdxg

struct cfdxg_mpnn {
    std::vector<float> host;   // FP32 master parameters (host mirror)
    cfdxg::DevBuf<float> params, grad, adam_m, adam_v, partial;
    cfdxg::DevBuf<__nv_bfloat16> wbf;   // per round: W1 (32x64) then W2 (32x32), BF16
    int64_t steps = 0;
    // binding
    const cfdxg_matrix* A = nullptr;
    int n = 0;
    cfdxg::DevBuf<float> ew, feats;
    cfdxg::DevBuf<int> gro, gco;   // off-diagonal couplings only (inference gather)
    cfdxg::DevBuf<float> gew;
    cfdxg::DevBuf<double> diag;
    // work
    cfdxg::DevBuf<float> H, AG, Z, dh, dh2, dhself, da, hA, hB, dyf;
    cfdxg::DevBuf<double> y, t, Ad, Ae, outb, w1, w2, q;
    cfdxg_amg* vcycle = nullptr;   // V-cycle the network is trained in front of
};

namespace cfdxg {
namespace {

using namespace mp;

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// x = [r/s, feats]; h0 = relu(W_in x + b_in).  Eight lanes per cell, each
// lane four features (one 16-byte store); the group's first lane forms r/s.
__global__ void k_encode(int n, const double* __restrict__ r, const double* __restrict__ rr,
                         const float* __restrict__ feats, const float* __restrict__ P, float* __restrict__ h) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int i = static_cast<int>(t >> 3), quarter = static_cast<int>(t & 7);
    const unsigned grp_mask = 0xffu << (threadIdx.x & 24);
    float x0 = 0.0f;
    if (i < n && quarter == 0) {
        const double s = sqrt(*rr / n);
        x0 = s > 0.0 ? static_cast<float>(r[i] / s) : 0.0f;
    }
    x0 = __shfl_sync(grp_mask, x0, 0, 8);
    if (i >= n) return;
    const float fv = feats[i], fp = feats[n + i], fd = feats[2 * n + i];
    const float* W = P + OFF_WIN;
    float o[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int f = 4 * quarter + q;
        const float pre = P[OFF_BIN + f] + W[f * 4 + 0] * x0 + W[f * 4 + 1] * fv + W[f * 4 + 2] * fp +
                          W[f * 4 + 3] * fd;
        o[q] = fmaxf(pre, 0.0f);
    }
    reinterpret_cast<float4*>(h)[static_cast<size_t>(i) * (F / 4) + quarter] = make_float4(o[0], o[1], o[2], o[3]);
}

// a_i = sum_k ew[k] h[co[k]]  (ew = 0 on the diagonal).  Warp per cell, lane = feature.
__global__ void k_gather(int n, const int* __restrict__ ro, const int* __restrict__ co, const float* __restrict__ ew,
                         const float* __restrict__ h, float* __restrict__ a) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= n) return;
    float s = 0.0f;
    for (int k = ro[w]; k < ro[w + 1]; ++k) s += ew[k] * h[static_cast<size_t>(co[k]) * F + lane];
    a[static_cast<size_t>(w) * F + lane] = s;
}

// One round's MLP (FP32): z = W1 [h, a] + b1; h_next = h + W2 relu(z) + b2.  Warp per cell.
__global__ void k_mlp_fwd(int n, const float* __restrict__ h, const float* __restrict__ a,
                          const float* __restrict__ Pr, float* __restrict__ z, float* __restrict__ hn) {
    __shared__ float W1[F][2 * F + 1];
    __shared__ float W2[F][F + 1];
    for (int q = threadIdx.x; q < F * 2 * F; q += blockDim.x) W1[q / (2 * F)][q % (2 * F)] = Pr[OFF_W1 + q];
    for (int q = threadIdx.x; q < F * F; q += blockDim.x) W2[q / F][q % F] = Pr[OFF_W2 + q];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * kWarps;
    for (int i = blockIdx.x * kWarps + (threadIdx.x >> 5); i < n; i += warps) {
        const float hv = h[static_cast<size_t>(i) * F + lane], av = a[static_cast<size_t>(i) * F + lane];
        float zz = Pr[OFF_B1 + lane];
        for (int m = 0; m < F; ++m) zz += W1[lane][m] * __shfl_sync(0xffffffffu, hv, m);
        for (int m = 0; m < F; ++m) zz += W1[lane][F + m] * __shfl_sync(0xffffffffu, av, m);
        const float g = fmaxf(zz, 0.0f);
        float z2 = Pr[OFF_B2 + lane];
        for (int q = 0; q < F; ++q) z2 += W2[lane][q] * __shfl_sync(0xffffffffu, g, q);
        z[static_cast<size_t>(i) * F + lane] = zz;
        hn[static_cast<size_t>(i) * F + lane] = hv + z2;
    }
}

// out_i = s (w_out . h_i + b_out) / a_ii.  Eight lanes per cell (16-byte loads),
// combined with a fixed butterfly.
__global__ void k_readout(int n, const float* __restrict__ h, const float* __restrict__ P, const double* rr,
                          const double* __restrict__ diag, double* __restrict__ out) {
    const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int i = static_cast<int>(t >> 3), quarter = static_cast<int>(t & 7);
    const unsigned grp_mask = 0xffu << (threadIdx.x & 24);
    float y = 0.0f;
    if (i < n) {
        const float4 v = reinterpret_cast<const float4*>(h)[static_cast<size_t>(i) * (F / 4) + quarter];
        const float* w = P + OFF_WOUT + 4 * quarter;
        y = w[0] * v.x + w[1] * v.y + w[2] * v.z + w[3] * v.w;
    }
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) y += __shfl_xor_sync(grp_mask, y, o, 8);
    if (i < n && quarter == 0) {
        const double s = sqrt(*rr / n);
        out[i] = s * static_cast<double>(y + P[OFF_BOUT]) / diag[i];
    }
}

// ---------------- fused tensor-core round (inference) ----------------
__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

constexpr int kUPad = 2 * F + 8;   // 72 bf16 per row: 144 B, keeps 4-byte loads conflict-light
constexpr int kW2Pad = F + 8;

// Inference round, gather-optimised.  A warp owns 16 consecutive cells.  Their
// off-diagonal couplings are one contiguous CSR segment, staged in shared
// memory with coalesced loads; the gather then runs 8 lanes per cell (each
// lane a 16-byte quarter-row of 4 features) over 4 cells at a time, with four
// neighbour rows in flight per lane.  [h, a] goes to shared memory as BF16 for
// the two tensor-core layers; the FP32 h stays in shared memory for the
// residual update.
constexpr int kTileCells = 16;
constexpr int kSegCap = 128;           // staged couplings per 16-cell tile
constexpr int kRoundWarps = 6;
constexpr int kRoundThreads = 32 * kRoundWarps;

// x_i = [r_i / s, f_V, f_P, f_D] packed as one float4 per cell (k_encode's
// input, 16 bytes), so the first round reads it instead of a 128-byte h0 row.
__global__ void k_pack_input(int n, const double* __restrict__ r, const double* __restrict__ rr,
                             const float* __restrict__ feats, float4* __restrict__ xin) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double s = sqrt(*rr / n);
    const float x0 = s > 0.0 ? static_cast<float>(r[i] / s) : 0.0f;
    xin[i] = make_float4(x0, feats[i], feats[n + i], feats[2 * n + i]);
}

// The first round's input state h0 = relu(W_in x + b_in), formed where the
// round reads it (k_encode's arithmetic) instead of being written by a
// separate kernel and read back: one lane's quarter-row (four features).
struct Encoder {
    const float4* xin;
    float w[4][4], b[4];
    __device__ __forceinline__ void load(const float4* xin_, const float* P, int quarter) {
        xin = xin_;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int f = 4 * quarter + q;
            b[q] = P[OFF_BIN + f];
#pragma unroll
            for (int c = 0; c < 4; ++c) w[q][c] = P[OFF_WIN + f * 4 + c];
        }
    }
    __device__ __forceinline__ float4 h0(int j) const {
        const float4 x = xin[j];
        float o[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            o[q] = fmaxf(b[q] + w[q][0] * x.x + w[q][1] * x.y + w[q][2] * x.z + w[q][3] * x.w, 0.0f);
        return make_float4(o[0], o[1], o[2], o[3]);
    }
};

// Gather of one 16-cell tile: sH = h (FP32), sU = [h, a] (BF16), a_i = sum_j w_ij h_j.
// Lanes 8q..8q+7 take cell 4 * pass + q, each lane one 16-byte quarter-row.
// STAGED: the tile's couplings are in sIdx / sW (index k - seg_b); otherwise
// they are read from global memory.  FIRST: h is the encoder's h0.
// BF16 -> FP32 is exact: the BF16 bits are the upper half of the FP32 word.
// Done with integer shifts and masks (the ALU), which measured faster here
// than the conversion instructions.
__device__ __forceinline__ float4 unpack_bf16x4(uint2 u) {
    return make_float4(__uint_as_float(u.x << 16), __uint_as_float(u.x & 0xffff0000u),
                       __uint_as_float(u.y << 16), __uint_as_float(u.y & 0xffff0000u));
}

template <bool STAGED, bool FIRST>
__device__ __forceinline__ void gather_tile(int c0, int cells, int rb, int re, int seg_b, const int* sIdx,
                                            const float* sW, const int* __restrict__ gco,
                                            const float* __restrict__ gew, const __nv_bfloat16* __restrict__ h_in,
                                            const Encoder& enc, float (*sH)[F], __nv_bfloat16 (*sU)[kUPad]) {
    const int lane = threadIdx.x & 31;
    // the state between rounds is BF16: a lane's quarter-row is 8 bytes
    const uint2* h8 = reinterpret_cast<const uint2*>(h_in);
    const int grp = lane >> 3, quarter = lane & 7;
    // 32-bit row offsets (the binding keeps n * F / 4 below 2^31)
    auto hrow = [&](int j) -> float4 {
        if constexpr (FIRST) return enc.h0(j);
        else return unpack_bf16x4(h8[j * (F / 4) + quarter]);
    };
    // the four passes unrolled: their neighbour rows are loaded together
#pragma unroll
    for (int pass = 0; pass < kTileCells / 4; ++pass) {
        const int r = pass * 4 + grp;
        const int b = __shfl_sync(0xffffffffu, rb, r), e = __shfl_sync(0xffffffffu, re, r);
        float4 hv = make_float4(0.f, 0.f, 0.f, 0.f), av = make_float4(0.f, 0.f, 0.f, 0.f);
        const int self = r < cells ? c0 + r : c0;
        if (r < cells) hv = hrow(self);
        // neighbours four at a time, the last group predicated (a tet cell has
        // at most four): the padding terms read the cell's own row with weight 0
        for (int k0 = b; k0 < e; k0 += 4) {
            int j[4];
            float w[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = k0 + u;
                const bool ok = k < e;
                j[u] = ok ? (STAGED ? sIdx[k - seg_b] : gco[k]) : self;
                w[u] = ok ? (STAGED ? sW[k - seg_b] : gew[k]) : 0.0f;
            }
            float4 v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = hrow(j[u]);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                av.x += w[u] * v[u].x; av.y += w[u] * v[u].y; av.z += w[u] * v[u].z; av.w += w[u] * v[u].w;
            }
        }
        *reinterpret_cast<float4*>(&sH[r][4 * quarter]) = hv;
        uint2 hp, ap;
        hp.x = pack_bf16(hv.x, hv.y); hp.y = pack_bf16(hv.z, hv.w);
        ap.x = pack_bf16(av.x, av.y); ap.y = pack_bf16(av.z, av.w);
        *reinterpret_cast<uint2*>(&sU[r][4 * quarter]) = hp;
        *reinterpret_cast<uint2*>(&sU[r][F + 4 * quarter]) = ap;
    }
}

// One round.  FIRST: the input state is formed from r by the encoder (no h0
// in memory).  LAST: the new state goes straight to the readout,
// out_i = s (w_out . h_i + b_out) / a_ii, instead of to h_out.
template <bool FIRST, bool LAST>
__global__ void __launch_bounds__(kRoundThreads) k_round_gather_tc(
    int n, const int* __restrict__ gro, const int* __restrict__ gco, const float* __restrict__ gew,
    const __nv_bfloat16* __restrict__ h_in, __nv_bfloat16* __restrict__ h_out, const __nv_bfloat16* __restrict__ W1g,
    const __nv_bfloat16* __restrict__ W2g, const float* __restrict__ Pr, const float* __restrict__ P,
    const double* __restrict__ r, const double* __restrict__ rr, const float* __restrict__ feats,
    const double* __restrict__ diag, double* __restrict__ yout) {
    __shared__ __align__(16) __nv_bfloat16 sW1[F][kUPad];
    __shared__ __align__(16) __nv_bfloat16 sW2[F][kW2Pad];
    __shared__ __align__(16) __nv_bfloat16 sU[kRoundWarps][kTileCells][kUPad];
    __shared__ __align__(16) float sH[kRoundWarps][kTileCells][F];
    __shared__ int sIdx[kRoundWarps][kSegCap];
    __shared__ float sW[kRoundWarps][kSegCap];
    __shared__ float sb1[F], sb2[F];
    for (int q = threadIdx.x; q < F * 2 * F; q += blockDim.x) sW1[q / (2 * F)][q % (2 * F)] = W1g[q];
    for (int q = threadIdx.x; q < F * F; q += blockDim.x) sW2[q / F][q % F] = W2g[q];
    if (threadIdx.x < F) {
        sb1[threadIdx.x] = Pr[OFF_B1 + threadIdx.x];
        sb2[threadIdx.x] = Pr[OFF_B2 + threadIdx.x];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Encoder enc;
    if constexpr (FIRST) enc.load(reinterpret_cast<const float4*>(feats), P, lane & 7);
    // persistent: each warp walks tiles with the grid's stride, the weights
    // staged once per block
    for (int tile = blockIdx.x * kRoundWarps + warp; tile * kTileCells < n; tile += gridDim.x * kRoundWarps) {
    const int c0 = tile * kTileCells;
    const int cells = min(kTileCells, n - c0);
    // tile segment of the coupling list
    const int seg_b = gro[c0], seg_e = gro[c0 + cells];
    const bool staged = seg_e - seg_b <= kSegCap;
    if (staged)
        for (int q = lane; q < seg_e - seg_b; q += 32) {
            sIdx[warp][q] = gco[seg_b + q];
            sW[warp][q] = gew[seg_b + q];
        }
    int rb = 0, re = 0;   // lanes 0..15: row range of cell c0 + lane
    if (lane < cells) {
        rb = gro[c0 + lane];
        re = gro[c0 + lane + 1];
    }
    __syncwarp();
    if (staged)
        gather_tile<true, FIRST>(c0, cells, rb, re, seg_b, sIdx[warp], sW[warp], gco, gew, h_in, enc, sH[warp],
                                 sU[warp]);
    else
        gather_tile<false, FIRST>(c0, cells, rb, re, seg_b, sIdx[warp], sW[warp], gco, gew, h_in, enc, sH[warp],
                                  sU[warp]);
    __syncwarp();
    const int g = lane >> 2, t = lane & 3;
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        acc[j][0] = sb1[8 * j + 2 * t];
        acc[j][1] = sb1[8 * j + 2 * t + 1];
        acc[j][2] = sb1[8 * j + 2 * t];
        acc[j][3] = sb1[8 * j + 2 * t + 1];
    }
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
        const uint32_t a0 = ld32(&sU[warp][g][16 * kk + 2 * t]);
        const uint32_t a1 = ld32(&sU[warp][g + 8][16 * kk + 2 * t]);
        const uint32_t a2 = ld32(&sU[warp][g][16 * kk + 2 * t + 8]);
        const uint32_t a3 = ld32(&sU[warp][g + 8][16 * kk + 2 * t + 8]);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t b0 = ld32(&sW1[8 * j + g][16 * kk + 2 * t]);
            const uint32_t b1 = ld32(&sW1[8 * j + g][16 * kk + 2 * t + 8]);
            mma_bf16(acc[j], a0, a1, a2, a3, b0, b1);
        }
    }
    uint32_t A2[2][4];
#pragma unroll
    for (int kk = 0; kk < 2; ++kk) {
        A2[kk][0] = pack_bf16(fmaxf(acc[2 * kk][0], 0.f), fmaxf(acc[2 * kk][1], 0.f));
        A2[kk][1] = pack_bf16(fmaxf(acc[2 * kk][2], 0.f), fmaxf(acc[2 * kk][3], 0.f));
        A2[kk][2] = pack_bf16(fmaxf(acc[2 * kk + 1][0], 0.f), fmaxf(acc[2 * kk + 1][1], 0.f));
        A2[kk][3] = pack_bf16(fmaxf(acc[2 * kk + 1][2], 0.f), fmaxf(acc[2 * kk + 1][3], 0.f));
    }
    float out[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int col = 8 * j + 2 * t;
        out[j][0] = sb2[col] + sH[warp][g][col];
        out[j][1] = sb2[col + 1] + sH[warp][g][col + 1];
        out[j][2] = sb2[col] + sH[warp][g + 8][col];
        out[j][3] = sb2[col + 1] + sH[warp][g + 8][col + 1];
    }
#pragma unroll
    for (int kk = 0; kk < 2; ++kk) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t b0 = ld32(&sW2[8 * j + g][16 * kk + 2 * t]);
            const uint32_t b1 = ld32(&sW2[8 * j + g][16 * kk + 2 * t + 8]);
            mma_bf16(out[j], A2[kk][0], A2[kk][1], A2[kk][2], A2[kk][3], b0, b1);
        }
    }
    const int rowa = g, rowb = g + 8;
    if constexpr (LAST) {
        // readout: row sums over this lane's columns, then across the 4 lanes of the row
        float ya = 0.0f, yb = 0.0f;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int col = 8 * j + 2 * t;
            const float w0 = P[OFF_WOUT + col], w1 = P[OFF_WOUT + col + 1];
            ya += w0 * out[j][0] + w1 * out[j][1];
            yb += w0 * out[j][2] + w1 * out[j][3];
        }
        ya += __shfl_xor_sync(0xffffffffu, ya, 1);
        ya += __shfl_xor_sync(0xffffffffu, ya, 2);
        yb += __shfl_xor_sync(0xffffffffu, yb, 1);
        yb += __shfl_xor_sync(0xffffffffu, yb, 2);
        if (t == 0) {
            const double s = sqrt(*rr / n);
            const float bo = P[OFF_BOUT];
            if (rowa < cells) yout[c0 + rowa] = s * static_cast<double>(ya + bo) / diag[c0 + rowa];
            if (rowb < cells) yout[c0 + rowb] = s * static_cast<double>(yb + bo) / diag[c0 + rowb];
        }
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int col = 8 * j + 2 * t;
            if (rowa < cells)
                *reinterpret_cast<uint32_t*>(&h_out[static_cast<size_t>(c0 + rowa) * F + col]) =
                    pack_bf16(out[j][0], out[j][1]);
            if (rowb < cells)
                *reinterpret_cast<uint32_t*>(&h_out[static_cast<size_t>(c0 + rowb) * F + col]) =
                    pack_bf16(out[j][2], out[j][3]);
        }
    }
    __syncwarp();   // the warp's sU / sH are rewritten by its next tile
    }
}

// ---------------- backward (FP32) ----------------
// loss pieces: d = e - out
__global__ void k_sub(int n, const double* __restrict__ e, const double* __restrict__ out, double* __restrict__ d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] = e[i] - out[i];
}

// dy = s * (-2 Ad / eAe) / a_ii
__global__ void k_dy(int n, const double* __restrict__ Ad, const double* eAe, const double* rr,
                     const double* __restrict__ diag, float* __restrict__ dy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double s = sqrt(*rr / n);
    dy[i] = static_cast<float>(s * (-2.0 * Ad[i] / *eAe) / diag[i]);
}

// Adds a per-warp accumulator row set (lane o owns `len` values) into the
// block's partial, warps in order; then adds the block total to partial[block].
__device__ void block_accumulate(float* acc_smem, const float* lane_vals, int len, int base, float* partial_block) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int w = 0; w < kWarps; ++w) {
        if (warp == w)
            for (int q = 0; q < len; ++q) {
                float& dst = acc_smem[lane * len + q];
                dst = (w == 0 ? 0.0f : dst) + lane_vals[q];
            }
        __syncthreads();
    }
    for (int q = threadIdx.x; q < F * len; q += blockDim.x) partial_block[base + q] += acc_smem[q];
    __syncthreads();
}

__global__ void k_readout_bwd(int n, const float* __restrict__ h, const float* __restrict__ dy,
                              const float* __restrict__ P, float* __restrict__ dh, float* __restrict__ partial) {
    __shared__ float sw[kWarps][F];
    __shared__ float sb[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float aw = 0.0f, ab = 0.0f;
    const int warps = gridDim.x * kWarps;
    for (int i = blockIdx.x * kWarps + warp; i < n; i += warps) {
        const float d = dy[i];
        dh[static_cast<size_t>(i) * F + lane] = P[OFF_WOUT + lane] * d;
        aw += d * h[static_cast<size_t>(i) * F + lane];
        ab += d;
    }
    sw[warp][lane] = aw;
    if (lane == 0) sb[warp] = ab;
    __syncthreads();
    float* pb = partial + static_cast<size_t>(blockIdx.x) * NP;
    if (threadIdx.x < F) {
        float s = 0.0f;
        for (int w = 0; w < kWarps; ++w) s += sw[w][threadIdx.x];
        pb[OFF_WOUT + threadIdx.x] += s;
    }
    if (threadIdx.x == 0) {
        float s = 0.0f;
        for (int w = 0; w < kWarps; ++w) s += sb[w];
        pb[OFF_BOUT] += s;
    }
}

// MLP backward of one round.  Inputs: h_k, a_k, z_k, dh (= dL/dh_{k+1}).
// Outputs: dhself = dL/dh_k through the MLP's h input, da = dL/da_k; weight
// gradients into this block's partial (round slots).
__global__ void __launch_bounds__(kThreads) k_mlp_bwd(int n, const float* __restrict__ h, const float* __restrict__ a,
                                                      const float* __restrict__ z, const float* __restrict__ dh,
                                                      const float* __restrict__ Pr, float* __restrict__ dhself,
                                                      float* __restrict__ da, float* __restrict__ partial,
                                                      int round_base) {
    __shared__ float W1[F][2 * F + 1];
    __shared__ float W2[F][F + 1];
    __shared__ float acc[F * (2 * F)];
    for (int q = threadIdx.x; q < F * 2 * F; q += blockDim.x) W1[q / (2 * F)][q % (2 * F)] = Pr[OFF_W1 + q];
    for (int q = threadIdx.x; q < F * F; q += blockDim.x) W2[q / F][q % F] = Pr[OFF_W2 + q];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    float gW1[2 * F], gW2[F], gb1 = 0.0f, gb2 = 0.0f;
#pragma unroll
    for (int q = 0; q < 2 * F; ++q) gW1[q] = 0.0f;
#pragma unroll
    for (int q = 0; q < F; ++q) gW2[q] = 0.0f;
    const int warps = gridDim.x * kWarps;
    for (int i = blockIdx.x * kWarps + (threadIdx.x >> 5); i < n; i += warps) {
        const size_t row = static_cast<size_t>(i) * F + lane;
        const float hv = h[row], av = a[row], zv = z[row], dz2 = dh[row];
        const float gv = fmaxf(zv, 0.0f);
        // lane o: dW2[o][q] += dz2[o] g[q]
#pragma unroll
        for (int q = 0; q < F; ++q) gW2[q] += dz2 * __shfl_sync(0xffffffffu, gv, q);
        gb2 += dz2;
        // lane q: dg[q] = sum_o W2[o][q] dz2[o]
        float dg = 0.0f;
        for (int o = 0; o < F; ++o) dg += W2[o][lane] * __shfl_sync(0xffffffffu, dz2, o);
        const float dz1 = zv > 0.0f ? dg : 0.0f;
#pragma unroll
        for (int m = 0; m < F; ++m) gW1[m] += dz1 * __shfl_sync(0xffffffffu, hv, m);
#pragma unroll
        for (int m = 0; m < F; ++m) gW1[F + m] += dz1 * __shfl_sync(0xffffffffu, av, m);
        gb1 += dz1;
        // lane m: du[m] = sum_q W1[q][m] dz1[q], du[32+m] likewise
        float du0 = 0.0f, du1 = 0.0f;
        for (int q = 0; q < F; ++q) {
            const float d = __shfl_sync(0xffffffffu, dz1, q);
            du0 += W1[q][lane] * d;
            du1 += W1[q][F + lane] * d;
        }
        dhself[row] = du0;
        da[row] = du1;
    }
    float* pb = partial + static_cast<size_t>(blockIdx.x) * NP + round_base;
    block_accumulate(acc, gW1, 2 * F, OFF_W1, pb);   // lane o's row o of dW1 -> [o*64 + m]
    block_accumulate(acc, gW2, F, OFF_W2, pb);
    float b1v[1] = {gb1}, b2v[1] = {gb2};
    block_accumulate(acc, b1v, 1, OFF_B1, pb);
    block_accumulate(acc, b2v, 1, OFF_B2, pb);
}

// dh_k[j] = dh[j] + dhself[j] + sum_i w_ji da[i]  (symmetric couplings: a gather)
__global__ void k_gather_bwd(int n, const int* __restrict__ ro, const int* __restrict__ co,
                             const float* __restrict__ ew, const float* __restrict__ dh,
                             const float* __restrict__ dhself, const float* __restrict__ da, float* __restrict__ out) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= n) return;
    float s = dh[static_cast<size_t>(w) * F + lane] + dhself[static_cast<size_t>(w) * F + lane];
    for (int k = ro[w]; k < ro[w + 1]; ++k) s += ew[k] * da[static_cast<size_t>(co[k]) * F + lane];
    out[static_cast<size_t>(w) * F + lane] = s;
}

__global__ void k_encode_bwd(int n, const double* __restrict__ r, const double* rr, const float* __restrict__ feats,
                             const float* __restrict__ h0, const float* __restrict__ dh, float* __restrict__ partial) {
    __shared__ float acc[F * 4];
    const int lane = threadIdx.x & 31;
    float gw[4] = {0.f, 0.f, 0.f, 0.f}, gb = 0.0f;
    const double s = sqrt(*rr / n);
    const int warps = gridDim.x * kWarps;
    for (int i = blockIdx.x * kWarps + (threadIdx.x >> 5); i < n; i += warps) {
        const size_t row = static_cast<size_t>(i) * F + lane;
        const float dpre = h0[row] > 0.0f ? dh[row] : 0.0f;
        const float x0 = s > 0.0 ? static_cast<float>(r[i] / s) : 0.0f;
        gw[0] += dpre * x0;
        gw[1] += dpre * feats[i];
        gw[2] += dpre * feats[n + i];
        gw[3] += dpre * feats[2 * n + i];
        gb += dpre;
    }
    float* pb = partial + static_cast<size_t>(blockIdx.x) * NP;
    block_accumulate(acc, gw, 4, OFF_WIN, pb);
    float bv[1] = {gb};
    block_accumulate(acc, bv, 1, OFF_BIN, pb);
}

__global__ void k_reduce_partials(const float* __restrict__ partial, int blocks, float scale, float* __restrict__ grad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NP) return;
    float s = 0.0f;
    for (int b = 0; b < blocks; ++b) s += partial[static_cast<size_t>(b) * NP + p];
    grad[p] = s * scale;
}

__global__ void k_adam(float* __restrict__ P, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       float lr, float bc1, float bc2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= NP) return;
    const float gi = g[p];
    m[p] = 0.9f * m[p] + 0.1f * gi;
    v[p] = 0.999f * v[p] + 0.001f * gi * gi;
    P[p] -= lr * (m[p] / bc1) / (sqrtf(v[p] / bc2) + 1e-8f);
}

__global__ void k_to_bf16(const float* __restrict__ P, __nv_bfloat16* __restrict__ wbf) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= R * 3 * F * F) return;
    const int r = q / (3 * F * F), k = q % (3 * F * F);
    const float* base = P + ROUND0 + r * ROUND_SIZE;
    wbf[q] = __float2bfloat16_rn(k < 2 * F * F ? base[OFF_W1 + k] : base[OFF_W2 + (k - 2 * F * F)]);
}

// learned composition helpers
__global__ void k_residual64(int n, const int* __restrict__ ro, const int* __restrict__ co,
                             const double* __restrict__ va, const double* __restrict__ v,
                             const double* __restrict__ y, double* __restrict__ t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double s = 0.0;
    for (int k = ro[i]; k < ro[i + 1]; ++k) s += va[k] * y[co[k]];
    t[i] = v[i] - s;
}

__global__ void k_add_inplace(int n, double* __restrict__ z, const double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) z[i] += y[i];
}

// ---------------- host helpers ----------------
void require_bound(const cfdxg_mpnn* net) {
    if (!net->A || net->n <= 0) throw Error(CFDXG_ERR_NOT_READY, "network is not bound to a matrix (cfdxg_mpnn_bind)");
}

void upload_params(cfdxg_context* ctx, cfdxg_mpnn* net) {
    net->params.upload(net->host, ctx->stream);
    net->wbf.resize(static_cast<size_t>(R) * 3 * F * F);
    k_to_bf16<<<blocks_for(R * 3 * F * F, 256), 256, 0, ctx->stream>>>(net->params.get(), net->wbf.get());
    check_launch(ctx);
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
}

double* scalar(cfdxg_context* ctx, int k) { return ctx->scratch.scalars + 3000 + k; }

// Inference: out = N(r) (tensor-core rounds).
void infer(cfdxg_context* ctx, cfdxg_mpnn* net, const double* r, double* out) {
    const int n = net->n;
    cudaStream_t s = ctx->stream;
    double* rr = scalar(ctx, 0);
    enqueue_dot(ctx, n, r, r, rr);
    // the packed first-round input x (16 bytes per cell) in the first quarter
    // of hA: the first round reads it and writes hB, and hA is next written by
    // the second round
    float4* xin = reinterpret_cast<float4*>(net->hA.get());
    {
        ProfScope ps(ctx, "mpnn_pack_input", (8.0 + 12.0 + 16.0) * n);
        k_pack_input<<<blocks_for(n, 256), 256, 0, s>>>(n, r, rr, net->feats.get(), xin);
        check_launch(ctx);
    }
    // the state between rounds is BF16 (64 bytes per cell: the 1.57 M-cell
    // state fits in L2, so the neighbour gathers hit it there)
    __nv_bfloat16* hin = reinterpret_cast<__nv_bfloat16*>(net->hA.get());
    __nv_bfloat16* hout = reinterpret_cast<__nv_bfloat16*>(net->hB.get());
    const int tiles = (n + kTileCells - 1) / kTileCells;
    for (int k = 0; k < R; ++k) {
        const __nv_bfloat16* w = net->wbf.get() + static_cast<size_t>(k) * 3 * F * F;
        const bool first = k == 0, last = k == R - 1;
        // compulsory bytes: the state read (r and the cell features in the
        // first round) and written (the output and diagonal in the last), the
        // coupling list once
        const double in_bytes = first ? 16.0 * n : 2.0 * F * n;
        const double out_bytes = last ? 16.0 * n : 2.0 * F * n;
        ProfScope ps(ctx, first ? "mpnn_round_first_tc" : (last ? "mpnn_round_last_tc" : "mpnn_round_gather_tc"),
                     in_bytes + out_bytes + 4.0 * (n + 1) + 8.0 * static_cast<double>(net->gco.size()));
        auto kern = first ? k_round_gather_tc<true, false>
                          : (last ? k_round_gather_tc<false, true> : k_round_gather_tc<false, false>);
        // persistent grid of five blocks per SM (the shared-memory limit) for
        // the middle and last rounds: 166 / 171 instead of 210 / 220 us at
        // 64^3.  The first round, which forms h0 per neighbour, measured
        // slower that way (277 vs 243 us) and takes one tile per warp.
        const int all = (tiles + kRoundWarps - 1) / kRoundWarps;
        const int grid = first ? all : std::min(all, 5 * ctx->sm_count);
        kern<<<grid, kRoundThreads, 0, s>>>(
            n, net->gro.get(), net->gco.get(), net->gew.get(), hin, hout, w, w + 2 * F * F,
            net->params.get() + ROUND0 + k * ROUND_SIZE, net->params.get(), r, rr,
            first ? reinterpret_cast<const float*>(xin) : nullptr, net->diag.get(), out);
        check_launch(ctx);
        std::swap(hin, hout);
    }
}

// Training forward for one sample; keeps activations in H, AG, Z.
void forward_train(cfdxg_context* ctx, cfdxg_mpnn* net, const double* r, double* out, double* rr) {
    const int n = net->n;
    cudaStream_t s = ctx->stream;
    const size_t st = static_cast<size_t>(n) * F;
    enqueue_dot(ctx, n, r, r, rr);
    k_encode<<<blocks_for(static_cast<int64_t>(n) * 8, 256), 256, 0, s>>>(n, r, rr, net->feats.get(),
                                                                          net->params.get(), net->H.get());
    check_launch(ctx);
    for (int k = 0; k < R; ++k) {
        k_gather<<<blocks_for(static_cast<int64_t>(n) * 32, 256), 256, 0, s>>>(
            n, net->A->ro.get(), net->A->co.get(), net->ew.get(), net->H.get() + k * st, net->AG.get() + k * st);
        check_launch(ctx);
        k_mlp_fwd<<<kGridBlocks, kThreads, 0, s>>>(n, net->H.get() + k * st, net->AG.get() + k * st,
                                                   net->params.get() + ROUND0 + k * ROUND_SIZE, net->Z.get() + k * st,
                                                   net->H.get() + (k + 1) * st);
        check_launch(ctx);
    }
    k_readout<<<blocks_for(static_cast<int64_t>(n) * 8, 256), 256, 0, s>>>(n, net->H.get() + R * st,
                                                                            net->params.get(), rr, net->diag.get(), out);
    check_launch(ctx);
}

// Loss and gradient (accumulated into net->partial) for one pair; returns the loss.
double loss_grad_one(cfdxg_context* ctx, cfdxg_mpnn* net, const double* r, const double* e) {
    const int n = net->n;
    cudaStream_t s = ctx->stream;
    const size_t st = static_cast<size_t>(n) * F;
    double* rr = scalar(ctx, 1);
    double* eAe = scalar(ctx, 2);
    double* dAd = scalar(ctx, 3);
    forward_train(ctx, net, r, net->outb.get(), rr);
    k_sub<<<blocks_for(n, 256), 256, 0, s>>>(n, e, net->outb.get(), net->t.get());
    check_launch(ctx);
    spmv_fp64(ctx, net->A, net->t.get(), net->Ad.get());
    spmv_fp64(ctx, net->A, e, net->Ae.get());
    if (!net->vcycle) {
        enqueue_dot(ctx, n, e, net->Ae.get(), eAe);
        enqueue_dot(ctx, n, net->t.get(), net->Ad.get(), dAd);
    } else {
        // w1 = E d, w2 = E w1 (E = I - M A); gradient direction A w2; scale by ||E e||_A^2
        amg_apply_device(ctx, net->vcycle, net->Ad.get(), net->q.get());
        k_sub<<<blocks_for(n, 256), 256, 0, s>>>(n, net->t.get(), net->q.get(), net->w1.get());
        check_launch(ctx);
        spmv_fp64(ctx, net->A, net->w1.get(), net->Ad.get());            // A w1
        enqueue_dot(ctx, n, net->w1.get(), net->Ad.get(), dAd);
        amg_apply_device(ctx, net->vcycle, net->Ad.get(), net->q.get());
        k_sub<<<blocks_for(n, 256), 256, 0, s>>>(n, net->w1.get(), net->q.get(), net->w2.get());
        check_launch(ctx);
        spmv_fp64(ctx, net->A, net->w2.get(), net->Ad.get());            // A w2
        amg_apply_device(ctx, net->vcycle, net->Ae.get(), net->q.get());  // M A e
        k_sub<<<blocks_for(n, 256), 256, 0, s>>>(n, e, net->q.get(), net->w1.get());   // E e
        check_launch(ctx);
        spmv_fp64(ctx, net->A, net->w1.get(), net->Ae.get());
        enqueue_dot(ctx, n, net->w1.get(), net->Ae.get(), eAe);
    }
    k_dy<<<blocks_for(n, 256), 256, 0, s>>>(n, net->Ad.get(), eAe, rr, net->diag.get(), net->dyf.get());
    check_launch(ctx);
    k_readout_bwd<<<kGridBlocks, kThreads, 0, s>>>(n, net->H.get() + R * st, net->dyf.get(), net->params.get(),
                                                   net->dh.get(), net->partial.get());
    check_launch(ctx);
    float* dh = net->dh.get();
    float* dh2 = net->dh2.get();
    for (int k = R - 1; k >= 0; --k) {
        k_mlp_bwd<<<kGridBlocks, kThreads, 0, s>>>(n, net->H.get() + k * st, net->AG.get() + k * st,
                                                   net->Z.get() + k * st, dh, net->params.get() + ROUND0 + k * ROUND_SIZE,
                                                   net->dhself.get(), net->da.get(), net->partial.get(),
                                                   ROUND0 + k * ROUND_SIZE);
        check_launch(ctx);
        k_gather_bwd<<<blocks_for(static_cast<int64_t>(n) * 32, 256), 256, 0, s>>>(
            n, net->A->ro.get(), net->A->co.get(), net->ew.get(), dh, net->dhself.get(), net->da.get(), dh2);
        check_launch(ctx);
        std::swap(dh, dh2);
    }
    k_encode_bwd<<<kGridBlocks, kThreads, 0, s>>>(n, r, rr, net->feats.get(), net->H.get(), dh, net->partial.get());
    check_launch(ctx);
    double h[2];
    CFDXG_CUDA(cudaMemcpyAsync(h, eAe, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CFDXG_CUDA(cudaStreamSynchronize(s));
    return h[1] / h[0];
}

double loss_grad_batch(cfdxg_context* ctx, cfdxg_mpnn* net, const double* r, const double* e, int batch) {
    require_bound(net);
    if (net->vcycle && net->vcycle->host.levels.front().A.n != net->n)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "training V-cycle and bound matrix differ in size");
    const int n = net->n;
    net->partial.resize(static_cast<size_t>(kGridBlocks) * NP);
    net->partial.zero(ctx->stream);
    net->grad.resize(NP);
    double total = 0.0;
    for (int b = 0; b < batch; ++b)
        total += loss_grad_one(ctx, net, r + static_cast<size_t>(b) * n, e + static_cast<size_t>(b) * n);
    k_reduce_partials<<<blocks_for(NP, 256), 256, 0, ctx->stream>>>(net->partial.get(), kGridBlocks,
                                                                    1.0f / static_cast<float>(batch), net->grad.get());
    check_launch(ctx);
    return total / batch;
}

uint64_t fnv1a(const void* data, size_t bytes) {
    const auto* p = static_cast<const unsigned char*>(data);
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < bytes; ++i) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

}  // namespace

void bind_learned_to_matrix(cfdxg_context*, cfdxg_mpnn* net, const cfdxg_matrix* A) {
    if (!net->A || net->A != A)
        throw Error(CFDXG_ERR_NOT_READY, "the learned network is not bound to this matrix (cfdxg_mpnn_bind)");
}

bool learned_then_amg(cfdxg_context* ctx, cfdxg_mpnn* net, const cfdxg_matrix* A, const double* v, double* z,
                      const std::function<void(const double*, double*)>& amg, int64_t*) {
    const int n = net->n;
    cudaStream_t s = ctx->stream;
    infer(ctx, net, v, net->y.get());
    k_residual64<<<blocks_for(n, 256), 256, 0, s>>>(n, A->ro.get(), A->co.get(), A->va.get(), v, net->y.get(),
                                                     net->t.get());
    check_launch(ctx);
    amg(net->t.get(), z);
    k_add_inplace<<<blocks_for(n, 256), 256, 0, s>>>(n, z, net->y.get());
    check_launch(ctx);
    return true;
}

}  // namespace cfdxg

using namespace cfdxg;

extern "C" int cfdxg_mpnn_create(cfdxg_context* ctx, uint64_t seed, cfdxg_mpnn** out) {
    if (!ctx || !out) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    auto net = std::make_unique<cfdxg_mpnn>();
    net->host.assign(mp::NP, 0.0f);
    std::mt19937_64 g(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    auto fill = [&](int off, int rows, int cols) {
        const double sc = std::sqrt(1.0 / cols);
        for (int q = 0; q < rows * cols; ++q) net->host[off + q] = static_cast<float>(nd(g) * sc);
    };
    fill(mp::OFF_WIN, mp::F, 4);
    for (int k = 0; k < mp::R; ++k) {
        fill(mp::ROUND0 + k * mp::ROUND_SIZE + mp::OFF_W1, mp::F, 2 * mp::F);
        fill(mp::ROUND0 + k * mp::ROUND_SIZE + mp::OFF_W2, mp::F, mp::F);
    }
    for (int q = 0; q < mp::F; ++q) net->host[mp::OFF_WOUT + q] = static_cast<float>(0.1 * nd(g));
    net->adam_m.resize(mp::NP);
    net->adam_v.resize(mp::NP);
    net->adam_m.zero(ctx->stream);
    net->adam_v.zero(ctx->stream);
    upload_params(ctx, net.get());
    *out = net.release();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_mpnn_destroy(cfdxg_mpnn* net) {
    delete net;
    return CFDXG_OK;
}

extern "C" int cfdxg_mpnn_num_parameters(const cfdxg_mpnn* net, int64_t* count) {
    if (!net || !count) return CFDXG_ERR_INVALID_ARGUMENT;
    *count = mp::NP;
    return CFDXG_OK;
}

extern "C" int cfdxg_mpnn_get_parameters(cfdxg_context* ctx, const cfdxg_mpnn* net, float* params) {
    if (!ctx || !net || !params) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    net->params.download(params, ctx->stream);
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_mpnn_set_parameters(cfdxg_context* ctx, cfdxg_mpnn* net, const float* params) {
    if (!ctx || !net || !params) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    net->host.assign(params, params + mp::NP);
    upload_params(ctx, net);
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_mpnn_save(cfdxg_context* ctx, const cfdxg_mpnn* net, const char* path) {
    if (!ctx || !net || !path) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    std::vector<float> p(mp::NP);
    net->params.download(p.data(), ctx->stream);
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    FILE* f = std::fopen(path, "wb");
    if (!f) throw Error(CFDXG_ERR_IO, std::string("cannot open ") + path);
    const char magic[8] = {'C', 'F', 'D', 'X', 'M', 'P', 'N', 'N'};
    const uint32_t version = 1, count = mp::NP;
    const uint64_t sum = fnv1a(p.data(), p.size() * sizeof(float));
    bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(&version, 4, 1, f) == 1 &&
              std::fwrite(&count, 4, 1, f) == 1 && std::fwrite(p.data(), sizeof(float), p.size(), f) == p.size() &&
              std::fwrite(&sum, 8, 1, f) == 1;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) throw Error(CFDXG_ERR_IO, std::string("cannot write ") + path);
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_mpnn_load(cfdxg_context* ctx, cfdxg_mpnn* net, const char* path) {
    if (!ctx || !net || !path) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    FILE* f = std::fopen(path, "rb");
    if (!f) throw Error(CFDXG_ERR_IO, std::string("cannot open ") + path);
    char magic[8];
    uint32_t version = 0, count = 0;
    uint64_t sum = 0;
    std::vector<float> p(mp::NP);
    const bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "CFDXMPNN", 8) == 0 &&
                    std::fread(&version, 4, 1, f) == 1 && version == 1 && std::fread(&count, 4, 1, f) == 1 &&
                    count == static_cast<uint32_t>(mp::NP) &&
                    std::fread(p.data(), sizeof(float), p.size(), f) == p.size() && std::fread(&sum, 8, 1, f) == 1;
    std::fclose(f);
    if (!ok) throw Error(CFDXG_ERR_IO, std::string("not a network weight file: ") + path);
    if (sum != fnv1a(p.data(), p.size() * sizeof(float))) throw Error(CFDXG_ERR_IO, "weight file checksum mismatch");
    net->host = p;
    upload_params(ctx, net);
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_mpnn_bind(cfdxg_context* ctx, cfdxg_mpnn* net, cfdxg_mesh* mesh, const cfdxg_matrix* A,
                               const double* a_P, int32_t mem) {
    if (!ctx || !net || !mesh || !A || !a_P) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    check_mem_flag(mem);
    if (!mesh->geometry_ready) throw Error(CFDXG_ERR_NOT_READY, "geometry not built");
    if (A->n != mesh->n_cells) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "matrix and mesh sizes differ");
    // inference addresses the state with 32-bit row offsets (n * F / 4 quarter-rows)
    if (A->n > std::numeric_limits<int>::max() / mp::F)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "mesh too large for the learned stage");
    auto* M = const_cast<cfdxg_matrix*>(A);
    matrix_sync_host_values(ctx, M);
    const int64_t n = A->n;
    const HostCsr& H = M->host;
    // per-row work on the host threads (every value is formed as before; only
    // the sums of the feature standardisation stay sequential, in row order)
    const auto rows = [n](auto&& fn) {
        const int workers = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(host_threads(), n / 65536)));
        if (workers <= 1) { fn(int64_t(0), n); return; }
        std::vector<std::thread> pool;
        for (int w = 0; w < workers; ++w) pool.emplace_back([&fn, n, w, workers] { fn(n * w / workers, n * (w + 1) / workers); });
        for (auto& t : pool) t.join();
    };
    std::vector<double> diag(n, 0.0), vol(n), ap(n);
    std::atomic<bool> bad_diag{false}, asymmetric{false}, bad_cell{false};
    rows([&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) {
            for (uint32_t k = H.ro[i]; k < H.ro[i + 1]; ++k)
                if (H.co[k] == i) diag[i] = H.va[k];
            if (!(diag[i] > 0.0)) bad_diag = true;
        }
    });
    if (bad_diag) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "the learned preconditioner needs a positive diagonal");
    // symmetric couplings are required (the backward pass gathers over the same graph)
    std::vector<float> ew(H.co.size(), 0.0f);
    std::vector<int> gro(n + 1, 0);
    rows([&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) {
            int off = 0;
            for (uint32_t k = H.ro[i]; k < H.ro[i + 1]; ++k) {
                const uint32_t j = H.co[k];
                if (j == i) continue;
                ++off;
                const uint32_t* lo = H.co.data() + H.ro[j];
                const uint32_t* hi = H.co.data() + H.ro[j + 1];
                const uint32_t* it = std::lower_bound(lo, hi, static_cast<uint32_t>(i));
                if (it == hi || *it != i || H.va[it - H.co.data()] != H.va[k]) {
                    asymmetric = true;
                    return;
                }
                ew[k] = static_cast<float>(-H.va[k] / std::sqrt(diag[i] * diag[j]));
            }
            gro[i + 1] = off;
        }
    });
    if (asymmetric) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "the learned preconditioner needs a symmetric matrix");
    mesh->cell_volume.download(vol.data(), ctx->stream);
    if (mem == CFDXG_MEM_DEVICE) CFDXG_CUDA(cudaMemcpyAsync(ap.data(), a_P, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    else std::memcpy(ap.data(), a_P, n * sizeof(double));
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<float> feats(3 * n);
    std::vector<double> logs(n);
    const auto standardise = [&](const std::vector<double>& v, int slot) {
        rows([&](int64_t b, int64_t e) { for (int64_t i = b; i < e; ++i) logs[i] = std::log(v[i]); });
        double mean = 0.0, sq = 0.0;
        for (int64_t i = 0; i < n; ++i) mean += logs[i];
        mean /= n;
        for (int64_t i = 0; i < n; ++i) sq += (logs[i] - mean) * (logs[i] - mean);
        const double sd = std::sqrt(sq / n);
        rows([&](int64_t b, int64_t e) {
            for (int64_t i = b; i < e; ++i)
                feats[slot * n + i] = static_cast<float>((logs[i] - mean) / (sd > 0.0 ? sd : 1.0));
        });
    };
    rows([&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i)
            if (!(vol[i] > 0.0) || !(ap[i] > 0.0)) bad_cell = true;
    });
    if (bad_cell) throw Error(CFDXG_ERR_INVALID_ARGUMENT, "volumes and a_P must be positive");
    standardise(vol, 0);
    standardise(ap, 1);
    standardise(diag, 2);
    net->ew.upload(ew, ctx->stream);
    // the coupling list without the diagonal: row offsets by a prefix sum, then rows in parallel
    for (int64_t i = 0; i < n; ++i) gro[i + 1] += gro[i];
    std::vector<int> gco(static_cast<std::size_t>(gro[n]));
    std::vector<float> gew(static_cast<std::size_t>(gro[n]));
    rows([&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) {
            int o = gro[i];
            for (uint32_t k = H.ro[i]; k < H.ro[i + 1]; ++k)
                if (H.co[k] != i) {
                    gco[o] = static_cast<int>(H.co[k]);
                    gew[o] = ew[k];
                    ++o;
                }
        }
    });
    net->gro.upload(gro, ctx->stream);
    net->gco.upload(gco, ctx->stream);
    net->gew.upload(gew, ctx->stream);
    net->feats.upload(feats, ctx->stream);
    net->diag.upload(diag, ctx->stream);
    const size_t st = static_cast<size_t>(n) * mp::F;
    net->H.resize(st * (mp::R + 1));
    net->AG.resize(st * mp::R);
    net->Z.resize(st * mp::R);
    net->dh.resize(st); net->dh2.resize(st); net->dhself.resize(st); net->da.resize(st);
    net->hA.resize(st); net->hB.resize(st); net->dyf.resize(n);
    net->y.resize(n); net->t.resize(n); net->Ad.resize(n); net->Ae.resize(n); net->outb.resize(n);
    net->w1.resize(n); net->w2.resize(n); net->q.resize(n);
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    net->A = A;
    net->n = static_cast<int>(n);
    ctx->error.clear();
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_mpnn_set_vcycle(cfdxg_context* ctx, cfdxg_mpnn* net, cfdxg_amg* amg) {
    if (!ctx || !net) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    if (amg && (!amg->ready || (!amg->d64 && !amg->d32)))
        throw Error(CFDXG_ERR_NOT_READY, "the V-cycle is not set up on the device");
    net->vcycle = amg;
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_mpnn_apply(cfdxg_context* ctx, cfdxg_mpnn* net, const double* r, double* y, int32_t mem) {
    if (!ctx || !net || !r || !y) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    NvtxRange nvtx_range("cfdxg.mpnn_apply");
    check_mem_flag(mem);
    require_bound(net);
    In<double> rin(ctx, r, net->n, mem);
    Out<double> yo(ctx, y, net->n, mem);
    infer(ctx, net, rin.get(), yo.get());
    yo.finish();
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_mpnn_loss_grad(cfdxg_context* ctx, cfdxg_mpnn* net, const double* r, const double* e,
                                    int32_t batch, int32_t mem, double* loss, float* grad) {
    if (!ctx || !net || !r || !e || batch <= 0) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    check_mem_flag(mem);
    require_bound(net);
    const int64_t total = static_cast<int64_t>(batch) * net->n;
    In<double> rin(ctx, r, total, mem), ein(ctx, e, total, mem);
    const double L = loss_grad_batch(ctx, net, rin.get(), ein.get(), batch);
    if (loss) *loss = L;
    if (grad) net->grad.download(grad, ctx->stream);
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}

extern "C" int cfdxg_mpnn_train_step(cfdxg_context* ctx, cfdxg_mpnn* net, const double* r, const double* e,
                                     int32_t batch, float lr, int32_t mem, double* loss) {
    if (!ctx || !net || !r || !e || batch <= 0 || !(lr > 0.0f)) return CFDXG_ERR_INVALID_ARGUMENT;
    CFDXG_GUARD_BEGIN
    check_mem_flag(mem);
    require_bound(net);
    const int64_t total = static_cast<int64_t>(batch) * net->n;
    In<double> rin(ctx, r, total, mem), ein(ctx, e, total, mem);
    const double L = loss_grad_batch(ctx, net, rin.get(), ein.get(), batch);
    ++net->steps;
    const float bc1 = 1.0f - std::pow(0.9f, static_cast<float>(net->steps));
    const float bc2 = 1.0f - std::pow(0.999f, static_cast<float>(net->steps));
    k_adam<<<blocks_for(mp::NP, 256), 256, 0, ctx->stream>>>(net->params.get(), net->grad.get(), net->adam_m.get(),
                                                             net->adam_v.get(), lr, bc1, bc2);
    check_launch(ctx);
    k_to_bf16<<<blocks_for(mp::R * 3 * mp::F * mp::F, 256), 256, 0, ctx->stream>>>(net->params.get(), net->wbf.get());
    check_launch(ctx);
    CFDXG_CUDA(cudaStreamSynchronize(ctx->stream));
    if (loss) *loss = L;
    return CFDXG_OK;
    CFDXG_GUARD_END(ctx)
}
