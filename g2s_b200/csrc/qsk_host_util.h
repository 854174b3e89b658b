// Host-side helpers shared by the host engines (qsk_host.cpp, qsk_tensor.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace qsk {

// device buffer owned by the host object that holds it
template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc(&p, sizeof(T) * count);
        if (e == cudaSuccess) n = count;
        else p = nullptr;
        return e;
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
