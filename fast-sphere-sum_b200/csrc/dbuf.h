// dbuf.h -- a device buffer that grows on demand (private to the library).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

namespace fss {

struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t ensure(size_t b) {
        if (b <= bytes && p) return cudaSuccess;
        release();
        if (b == 0) b = 16;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            p = nullptr;
            return e;
        }
        bytes = b;
        return cudaSuccess;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

}  // namespace fss
