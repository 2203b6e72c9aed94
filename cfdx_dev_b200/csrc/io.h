// io.h -- host/device argument staging and the C-ABI error guard.
#pragma once
#include <new>

#include "objects.h"

namespace cfdxg {

// A read-only array argument that may live on the host or the device.
template <class T>
class In {
public:
    In(cfdxg_context* ctx, const T* p, int64_t n, int32_t mem) {
        if (!p || n == 0) return;
        if (mem == CFDXG_MEM_DEVICE) {
            ptr_ = p;
        } else {
            buf_.upload(p, static_cast<std::size_t>(n), ctx->stream);
            ptr_ = buf_.get();
        }
    }
    const T* get() const { return ptr_; }

private:
    DevBuf<T> buf_;
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
            if (preload) buf_.upload(p, static_cast<std::size_t>(n), ctx->stream);
            else buf_.resize(static_cast<std::size_t>(n));
            ptr_ = buf_.get();
        }
    }
    T* get() const { return ptr_; }
    void finish() {
        if (host_ && mem_ != CFDXG_MEM_DEVICE && n_) {
            buf_.download(host_, ctx_->stream);
        }
    }

private:
    cfdxg_context* ctx_;
    T* host_;
    int64_t n_;
    int32_t mem_;
    DevBuf<T> buf_;
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
