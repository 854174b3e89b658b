// Host-side helpers shared by the host engines (qsk_host.cpp, qsk_tensor.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <utility>

namespace qsk {

// Device blocks kept across simulations, per device (qsk_host.cpp).  A
// simulation's buffers are handed here by qsk_sim_destroy after a device
// synchronisation, so no work in flight reads them; DBuf::alloc takes the
// smallest kept block of the current device that holds the request (and at
// most twice it, plus 2 MiB) before it calls cudaMalloc.  Blocks are not
// cleared: every buffer is written before it is read, as with cudaMalloc.
void *block_take(size_t bytes, size_t *cap);
bool block_keep(void *p, size_t cap);   // false: over the limit, the caller frees
extern thread_local bool g_keep_blocks; // set while qsk_sim_destroy releases

// device buffer owned by the host object that holds it
template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    size_t cap = 0;   // bytes of the block
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p && !(g_keep_blocks && block_keep(p, cap))) cudaFree(p);
        p = nullptr;
        n = 0;
        cap = 0;
    }
    cudaError_t alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        const size_t want = sizeof(T) * count;
        if (void *q = block_take(want, &cap)) {
            p = static_cast<T *>(q);
            n = count;
            return cudaSuccess;
        }
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) {
            n = count;
            cap = want;
        } else {
            p = nullptr;
        }
        return e;
    }
    void swap(DBuf &o) {
        std::swap(p, o.p);
        std::swap(n, o.n);
        std::swap(cap, o.cap);
    }
    cudaError_t ensure(size_t count) { return count <= n ? cudaSuccess : alloc(count); }
    cudaError_t upload(const T *h, size_t count, cudaStream_t st) {
        cudaError_t e = ensure(count);
        if (e != cudaSuccess) return e;
        return cudaMemcpyAsync(p, h, sizeof(T) * count, cudaMemcpyHostToDevice, st);
    }
};

// makes `dev` current for the scope of the guard
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace qsk

// return the calling thread's error (qsk_last_error) on a CUDA failure
#define QSK_CK(expr)                                                                                      \
    do {                                                                                                  \
        cudaError_t e_ = (expr);                                                                          \
        if (e_ != cudaSuccess) {                                                                          \
            int code_ = (e_ == cudaErrorMemoryAllocation) ? QSK_ERR_NOMEM : QSK_ERR_CUDA;                  \
            return ::qsk::set_error(code_, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__,       \
                                    __LINE__);                                                            \
        }                                                                                                 \
    } while (0)
