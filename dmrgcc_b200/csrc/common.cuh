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

// Process-wide count of the kernels this library has launched (read through
// dmrg_launch_count).  Every launch site is written `DMRG_LAUNCH kernel<<<...>>>(...)`.
void count_launch();
#define DMRG_LAUNCH ::dmrg::count_launch(),

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

// Stream-ordered pooled allocation.  While an AllocScope is alive on a thread,
// every DeviceBuffer that thread allocates comes from a per-device memory pool
// that keeps freed blocks (cudaMallocFromPoolAsync / cudaFreeAsync on the
// scope's stream): a sweep that rebuilds its tensors at every step then pays
// neither cudaMalloc nor the device-wide synchronisation of cudaFree each time.
// Work that touches such a buffer must be ordered after its allocation on that
// stream (all library work of one context runs on the context's stream).
class AllocScope {
public:
    explicit AllocScope(cudaStream_t st);
    ~AllocScope();
    AllocScope(const AllocScope&) = delete;
    AllocScope& operator=(const AllocScope&) = delete;

private:
    bool prev_active_;
    cudaStream_t prev_stream_;
};
// Reads and clears the context's device status word (waits for the stream);
// returns DMRG_OK or the code a kernel recorded (for example a bounded wait that
// timed out).
int take_device_status(dmrg_ctx_t ctx);
// The innermost scope's stream, or false when none is active on this thread.
bool alloc_scope(cudaStream_t* st);
// cudaMallocFromPoolAsync on the current device's pool (created on first use,
// release threshold unlimited so freed blocks stay cached for reuse).
cudaError_t pool_malloc(void** ptr, size_t bytes, cudaStream_t st);

// A device allocation owned by RAII; never copied.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    bool pooled = false;              // from the pool: freed on `stream`, in stream order
    cudaStream_t stream = nullptr;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), bytes(o.bytes), pooled(o.pooled), stream(o.stream) {
        o.ptr = nullptr;
        o.bytes = 0;
        o.pooled = false;
    }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        if (this != &o) {
            release();
            ptr = o.ptr;
            bytes = o.bytes;
            pooled = o.pooled;
            stream = o.stream;
            o.ptr = nullptr;
            o.bytes = 0;
            o.pooled = false;
        }
        return *this;
    }
    ~DeviceBuffer() { release(); }
    void release() {
        if (ptr) {
            if (pooled) cudaFreeAsync(ptr, stream);
            else cudaFree(ptr);
        }
        ptr = nullptr;
        bytes = 0;
        pooled = false;
    }
    int alloc(size_t n) {
        if (n <= bytes && ptr) return DMRG_OK;
        release();
        if (n == 0) return DMRG_OK;
        cudaStream_t st = nullptr;
        const bool pool = alloc_scope(&st);
        cudaError_t e = pool ? pool_malloc(&ptr, n, st) : cudaMalloc(&ptr, n);
        if (e != cudaSuccess) {
            ptr = nullptr;
            return set_error(DMRG_E_NOMEM, "%s(%zu) failed: %s", pool ? "cudaMallocFromPoolAsync" : "cudaMalloc", n,
                             cudaGetErrorString(e));
        }
        bytes = n;
        pooled = pool;
        stream = st;
        return DMRG_OK;
    }
    // Zero-fills the buffer, ordered like its allocation.
    int zero() {
        if (!ptr) return DMRG_OK;
        const cudaError_t e = pooled ? cudaMemsetAsync(ptr, 0, bytes, stream) : cudaMemset(ptr, 0, bytes);
        return e == cudaSuccess ? DMRG_OK : set_error(DMRG_E_CUDA, "cudaMemset: %s", cudaGetErrorString(e));
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
    // Pinned host words for small per-iteration device->host reads (Lanczos
    // convergence flags); one context is used by one host thread at a time.
    int* h_pinned = nullptr;
};
