// fm_devbuf.hpp — a growable device buffer owned by the host code.
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

namespace fm {

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    // (re)allocate to at least count elements; contents undefined
    cudaError_t reserve(size_t count) {
        if (count <= n && p) return cudaSuccess;
        release();
        if (count == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            return e;
        }
        n = count;
        return cudaSuccess;
    }
};

}  // namespace fm
