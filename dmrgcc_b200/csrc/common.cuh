// Shared internals of libdmrg_b200: error reporting, the context object and
// small device helpers.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "dmrg_b200.h"

namespace dmrg {

// Sets the thread's last-error message and returns `code`.
int set_error(int code, const char* fmt, ...);

#define DMRG_CUDA_TRY(expr)                                                                   \
    do {                                                                                      \
        cudaError_t err_ = (expr);                                                            \
        if (err_ != cudaSuccess)                                                              \
            return ::dmrg::set_error(DMRG_E_CUDA, "%s failed: %s (%s:%d)", #expr,             \
                                     cudaGetErrorString(err_), __FILE__, __LINE__);           \
    } while (0)

#define DMRG_TRY(expr)                  \
    do {                                \
        int rc_ = (expr);               \
        if (rc_ != DMRG_OK) return rc_; \
    } while (0)

// A device allocation owned by RAII; never copied.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), bytes(o.bytes) {
        o.ptr = nullptr;
        o.bytes = 0;
    }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        if (this != &o) {
            release();
            ptr = o.ptr;
            bytes = o.bytes;
            o.ptr = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~DeviceBuffer() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    int alloc(size_t n) {
        if (n <= bytes && ptr) return DMRG_OK;
        release();
        if (n == 0) return DMRG_OK;
        cudaError_t e = cudaMalloc(&ptr, n);
        if (e != cudaSuccess) {
            ptr = nullptr;
            return set_error(DMRG_E_NOMEM, "cudaMalloc(%zu) failed: %s", n, cudaGetErrorString(e));
        }
        bytes = n;
        return DMRG_OK;
    }
    template <class T>
    T* as() const { return static_cast<T*>(ptr); }
};

// Uploads a host vector into a DeviceBuffer on `stream` (synchronous w.r.t. the
// host vector: the copy completes before return).
template <class T>
int upload(DeviceBuffer& buf, const std::vector<T>& v, cudaStream_t stream) {
    DMRG_TRY(buf.alloc(v.size() * sizeof(T)));
    if (v.empty()) return DMRG_OK;
    DMRG_CUDA_TRY(cudaMemcpyAsync(buf.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    DMRG_CUDA_TRY(cudaStreamSynchronize(stream));
    return DMRG_OK;
}

}  // namespace dmrg

struct dmrg_ctx_s {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int num_sms = 148;
    // Device-side error word: kernels with iteration caps write a nonzero code.
    int* d_status = nullptr;
};
