// device.cuh -- shared device utilities of libcfdxg: the context, RAII device
// buffers, launch accounting and deterministic block reductions.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/cfdxg.h"

namespace cfdxg {

// Thrown inside the library, converted to a status code at the C ABI.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CFDXG_CUDA(call)                                                                  \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            throw ::cfdxg::Error(e_ == cudaErrorMemoryAllocation ? CFDXG_ERR_OUT_OF_MEMORY \
                                                                 : CFDXG_ERR_CUDA,        \
                                 std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)

// Programmatic dependent launch (sm_90+): a kernel launched with launch_pdl
// may be scheduled while its predecessor on the stream drains.  It lets its
// own dependents schedule early (pdl_trigger) and waits for the predecessor's
// completion and memory flush (pdl_wait) before it reads anything the
// predecessor wrote.  Both are no-ops for an ordinary launch.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_entry() {
    pdl_trigger();
    pdl_wait();
}

template <typename... KArgs, typename... Args>
inline void launch_pdl(cudaStream_t stream, void (*kern)(KArgs...), dim3 grid, dim3 block, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr{};
    attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr.val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    CFDXG_CUDA(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
}

constexpr int kReduceThreads = 256;
constexpr int kMaxReduceBlocks = 1184;  // 8 x 148 SMs: fixed partition => deterministic sums

// Device-side scratch owned by a context: reduction partials, tickets, a
// status word for device-detected errors, and pinned host mirrors.
struct Scratch {
    double* partial = nullptr;      // kMaxReduceBlocks * 4
    unsigned* ticket = nullptr;     // 8 tickets
    double* scalars = nullptr;      // 4096 device scalars (dots, norms, H columns)
    int* status = nullptr;          // device error word
    double* host_scalars = nullptr; // pinned mirror of `scalars`
    int* host_status = nullptr;     // pinned
};

// Reusable device staging buffers for host-memory arguments (avoids a
// cudaMalloc / cudaFree pair per call).
struct StagingPool {
    struct Entry {
        void* ptr = nullptr;
        std::size_t bytes = 0;
        bool in_use = false;
    };
    std::vector<Entry> entries;
};

struct KernelStats {
    std::string name;
    int64_t launches = 0;
    double ms = 0.0;
    double bytes = 0.0;
};

struct Profiler {
    bool on = false;
    struct Pending {
        int idx;
        cudaEvent_t a, b;
        double bytes;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    std::vector<KernelStats> stats;
};

}  // namespace cfdxg

struct cfdxg_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string error;
    std::string plan_reason;   // plan of the last solve_linear_system
    int64_t launches = 0;
    cfdxg::Scratch scratch;
    int sm_count = 148;
    std::shared_ptr<void> krylov_workspace;   // grown on demand by the Krylov driver
    cfdxg::Profiler prof;
    cfdxg::StagingPool staging;
};

namespace cfdxg {

// NVTX range over one library call: phases show up by name in Nsight
// timelines and can filter ncu captures; without a tool attached the calls do
// nothing.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

inline void count_launch(cfdxg_context* ctx, int64_t n = 1) { ctx->launches += n; }

// Event bracket around one eager launch (no-op unless profiling is enabled).
int prof_begin(cfdxg_context* ctx, const char* name, double bytes);
void prof_end(cfdxg_context* ctx, int token);
void prof_flush(cfdxg_context* ctx);

struct ProfScope {
    cfdxg_context* ctx;
    int token;
    ProfScope(cfdxg_context* c, const char* name, double bytes) : ctx(c), token(prof_begin(c, name, bytes)) {}
    ~ProfScope() { prof_end(ctx, token); }
};

inline void check_launch(cfdxg_context* ctx) {
    count_launch(ctx);
    CFDXG_CUDA(cudaGetLastError());
}

template <class T>
class DevBuf {
public:
    DevBuf() = default;
    explicit DevBuf(std::size_t n) { resize(n); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void resize(std::size_t n) {
        if (n == n_) return;
        release();
        if (n) CFDXG_CUDA(cudaMalloc(&p_, n * sizeof(T)));
        n_ = n;
    }
    void upload(const T* h, std::size_t n, cudaStream_t s) {
        resize(n);
        if (n) CFDXG_CUDA(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T>& h, cudaStream_t s) { upload(h.data(), h.size(), s); }
    void download(T* h, cudaStream_t s) const {
        if (n_) CFDXG_CUDA(cudaMemcpyAsync(h, p_, n_ * sizeof(T), cudaMemcpyDeviceToHost, s));
    }
    void zero(cudaStream_t s) {
        if (n_) CFDXG_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
    }
    T* get() const { return p_; }
    std::size_t size() const { return n_; }
    void release() {
        if (p_) cudaFree(p_);
        p_ = nullptr;
        n_ = 0;
    }

private:
    T* p_ = nullptr;
    std::size_t n_ = 0;
};

inline int blocks_for(int64_t n, int threads) {
    return static_cast<int>((n + threads - 1) / threads);
}

inline int reduce_blocks(int64_t n) {
    const int64_t b = (n + kReduceThreads * 4 - 1) / (kReduceThreads * 4);
    return static_cast<int>(b < 1 ? 1 : (b > kMaxReduceBlocks ? kMaxReduceBlocks : b));
}

// ---- device helpers ----

template <class T>
__device__ __forceinline__ T block_sum(T v, T* smem) {
    // fixed-order tree: warp shuffles, then warp partials summed by warp 0
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    if (warp == 0) {
        v = lane < nw ? smem[lane] : T(0);
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();
    return v;
}

template <class T>
__device__ __forceinline__ T block_max(T v, T* smem) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    if (warp == 0) {
        v = lane < nw ? smem[lane] : T(0);
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    }
    __syncthreads();
    return v;
}

// Last-block-done: returns true in exactly one block, after every block's
// partial is visible.  The final combination then runs in block-index order,
// so the result does not depend on which block finished last.
__device__ __forceinline__ bool last_block(unsigned* ticket) {
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned t = atomicAdd(ticket, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (is_last) __threadfence();
    return is_last;
}

}  // namespace cfdxg
