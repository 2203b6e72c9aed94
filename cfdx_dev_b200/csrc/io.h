// io.h -- host/device argument staging and the C-ABI error guard.
#pragma once
#include <new>

#include "objects.h"

namespace cfdxg {

// Borrow a device buffer of at least `bytes` from the context's staging pool.
inline int stage_acquire(cfdxg_context* ctx, std::size_t bytes) {
    auto& E = ctx->staging.entries;
    int best = -1;
    for (int k = 0; k < static_cast<int>(E.size()); ++k)
        if (!E[k].in_use && E[k].bytes >= bytes && (best < 0 || E[k].bytes < E[best].bytes)) best = k;
    if (best < 0) {
        for (int k = 0; k < static_cast<int>(E.size()); ++k)
            if (!E[k].in_use) {   // grow an idle entry
                CFDXG_CUDA(cudaFreeAsync(E[k].ptr, ctx->stream));
                E[k].ptr = nullptr;
                CFDXG_CUDA(cudaMallocAsync(&E[k].ptr, bytes, ctx->stream));
                E[k].bytes = bytes;
                best = k;
                break;
            }
    }
    if (best < 0) {
        StagingPool::Entry e;
        CFDXG_CUDA(cudaMallocAsync(&e.ptr, bytes, ctx->stream));
        e.bytes = bytes;
        E.push_back(e);
        best = static_cast<int>(E.size()) - 1;
    }
    E[best].in_use = true;
    return best;
}

inline void stage_release(cfdxg_context* ctx, int slot) {
    if (slot >= 0) ctx->staging.entries[slot].in_use = false;
}

// A read-only array argument that may live on the host or the device.
template <class T>
class In {
public:
    In(cfdxg_context* ctx, const T* p, int64_t n, int32_t mem) : ctx_(ctx) {
        if (!p || n == 0) return;
        if (mem == CFDXG_MEM_DEVICE) {
            ptr_ = p;
        } else {
            slot_ = stage_acquire(ctx, sizeof(T) * static_cast<std::size_t>(n));
            T* d = static_cast<T*>(ctx->staging.entries[slot_].ptr);
            CFDXG_CUDA(cudaMemcpyAsync(d, p, sizeof(T) * n, cudaMemcpyHostToDevice, ctx->stream));
            ptr_ = d;
        }
    }
    ~In() { stage_release(ctx_, slot_); }
    In(const In&) = delete;
    In& operator=(const In&) = delete;
    const T* get() const { return ptr_; }

private:
    cfdxg_context* ctx_;
    int slot_ = -1;
    const T* ptr_ = nullptr;
};

// A writable array argument; host outputs are staged and copied back by finish().
template <class T>
class Out {
public:
    Out(cfdxg_context* ctx, T* p, int64_t n, int32_t mem, bool preload = false)
        : ctx_(ctx), host_(p), n_(n), mem_(mem) {
        if (!p || n == 0) return;
        if (mem == CFDXG_MEM_DEVICE) {
            ptr_ = p;
        } else {
            slot_ = stage_acquire(ctx, sizeof(T) * static_cast<std::size_t>(n));
            ptr_ = static_cast<T*>(ctx->staging.entries[slot_].ptr);
            if (preload) CFDXG_CUDA(cudaMemcpyAsync(ptr_, p, sizeof(T) * n, cudaMemcpyHostToDevice, ctx->stream));
        }
    }
    ~Out() { stage_release(ctx_, slot_); }
    Out(const Out&) = delete;
    Out& operator=(const Out&) = delete;
    T* get() const { return ptr_; }
    void finish() {
        if (host_ && mem_ != CFDXG_MEM_DEVICE && n_)
            CFDXG_CUDA(cudaMemcpyAsync(host_, ptr_, sizeof(T) * n_, cudaMemcpyDeviceToHost, ctx_->stream));
    }

private:
    cfdxg_context* ctx_;
    T* host_;
    int64_t n_;
    int32_t mem_;
    int slot_ = -1;
    T* ptr_ = nullptr;
};

inline void check_mem_flag(int32_t mem) {
    if (mem != CFDXG_MEM_HOST && mem != CFDXG_MEM_DEVICE)
        throw Error(CFDXG_ERR_INVALID_ARGUMENT, "mem must be CFDXG_MEM_HOST or CFDXG_MEM_DEVICE");
}

}  // namespace cfdxg

#define CFDXG_GUARD_BEGIN try {
#define CFDXG_GUARD_END(ctx)                                      \
    }                                                             \
    catch (const cfdxg::Error& e) {                               \
        if (ctx) (ctx)->error = e.what();                         \
        return e.code;                                            \
    }                                                             \
    catch (const std::bad_alloc&) {                               \
        if (ctx) (ctx)->error = "host allocation failed";         \
        return CFDXG_ERR_OUT_OF_MEMORY;                           \
    }                                                             \
    catch (const std::exception& e) {                             \
        if (ctx) (ctx)->error = e.what();                         \
        return CFDXG_ERR_INVALID_ARGUMENT;                        \
    }
