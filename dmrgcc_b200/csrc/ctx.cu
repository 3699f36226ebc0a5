// Context, error reporting and memory entry points of the C ABI.
#include <cstring>
#include <mutex>

#include "blocksparse.h"
#include "common.cuh"

namespace dmrg {

static thread_local std::string g_last_error = "no error";

int set_error(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int build_site_desc(SiteDesc& s, int nl, int nr, const int* phys, const dmrg_blocks_t* ket, int d, int lb, int rb,
                    const double* W) {
    if (nl <= 0 || nr <= 0 || !phys || !ket || d <= 0 || lb <= 0 || rb <= 0 || !W)
        return set_error(DMRG_E_ARG, "invalid site description (nl=%d nr=%d d=%d lb=%d rb=%d)", nl, nr, d, lb, rb);
    s.nl = nl;
    s.nr = nr;
    s.d = d;
    s.lb = lb;
    s.rb = rb;
    s.phys.assign(phys, phys + (size_t)nl * nr);
    s.W.assign(W, W + (size_t)lb * rb * d * d);
    if (!s.ket.assign(*ket)) return set_error(DMRG_E_ARG, "invalid ket block list");
    s.bphys.clear();
    for (int k = 0; k < s.ket.count(); ++k) {
        int l = s.ket.left[k], r = s.ket.right[k];
        if (l < 0 || l >= nl || r < 0 || r >= nr)
            return set_error(DMRG_E_ARG, "ket block %d has sectors (%d,%d) outside %dx%d", k, l, r, nl, nr);
        int p = s.p(l, r);
        if (p < 0 || p >= d)
            return set_error(DMRG_E_ARG, "ket block %d (%d,%d) has physics index %d", k, l, r, p);
        s.bphys.push_back(p);
    }
    return DMRG_OK;
}

int build_site_desc_blocks(SiteDesc& s, int nl, int nr, const int* block_phys, const dmrg_blocks_t* ket, int d,
                           int lb, int rb, const double* W) {
    if (nl <= 0 || nr <= 0 || !block_phys || !ket || d <= 0 || lb <= 0 || rb <= 0 || !W)
        return set_error(DMRG_E_ARG, "invalid site description (nl=%d nr=%d d=%d lb=%d rb=%d)", nl, nr, d, lb, rb);
    s.nl = nl;
    s.nr = nr;
    s.d = d;
    s.lb = lb;
    s.rb = rb;
    s.phys.clear();
    s.W.assign(W, W + (size_t)lb * rb * d * d);
    if (!s.ket.assign(*ket)) return set_error(DMRG_E_ARG, "invalid ket block list");
    s.bphys.assign(block_phys, block_phys + s.ket.count());
    for (int k = 0; k < s.ket.count(); ++k) {
        const int l = s.ket.left[k], r = s.ket.right[k], p = s.bphys[k];
        if (l < 0 || l >= nl || r < 0 || r >= nr)
            return set_error(DMRG_E_ARG, "ket block %d has sectors (%d,%d) outside %dx%d", k, l, r, nl, nr);
        if (p < 0 || p >= d) return set_error(DMRG_E_ARG, "ket block %d has physics index %d", k, p);
    }
    return DMRG_OK;
}

}  // namespace dmrg

namespace dmrg {
namespace {
struct ScopeState {
    bool active = false;
    cudaStream_t stream = nullptr;
};
thread_local ScopeState g_scope;
std::mutex g_pool_mutex;
cudaMemPool_t g_pools[64] = {};
}  // namespace

AllocScope::AllocScope(cudaStream_t st) : prev_active_(g_scope.active), prev_stream_(g_scope.stream) {
    g_scope.active = true;
    g_scope.stream = st;
}
AllocScope::~AllocScope() {
    g_scope.active = prev_active_;
    g_scope.stream = prev_stream_;
}

int take_device_status(dmrg_ctx_t ctx) {
    int code = 0;
    DMRG_CUDA_TRY(cudaMemcpyAsync(&code, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    DMRG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (code == 0) return DMRG_OK;
    DMRG_CUDA_TRY(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), ctx->stream));
    return set_error(code, "a device routine gave up waiting (status %d); its output is incomplete", code);
}

bool alloc_scope(cudaStream_t* st) {
    if (st) *st = g_scope.stream;
    return g_scope.active;
}

cudaError_t pool_malloc(void** ptr, size_t bytes, cudaStream_t st) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lock(g_pool_mutex);
        if (!g_pools[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            e = cudaMemPoolCreate(&g_pools[dev], &props);
            if (e != cudaSuccess) return e;
            uint64_t keep = UINT64_MAX;  // freed blocks stay in the pool
            e = cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
            if (e != cudaSuccess) return e;
        }
        pool = g_pools[dev];
    }
    return cudaMallocFromPoolAsync(ptr, bytes, pool, st);
}
}  // namespace dmrg

using namespace dmrg;

extern "C" {

const char* dmrg_version(void) { return "dmrg_b200 0.1 (sm_100a)"; }

const char* dmrg_last_error(void) { return g_last_error.c_str(); }


int dmrg_ctx_create(int device, dmrg_ctx_t* out) {
    if (!out) return set_error(DMRG_E_ARG, "null output pointer");
    *out = nullptr;
    int n = 0;
    DMRG_CUDA_TRY(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return set_error(DMRG_E_ARG, "device %d out of range (%d devices)", device, n);
    DMRG_CUDA_TRY(cudaSetDevice(device));
    auto* c = new dmrg_ctx_s();
    c->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return set_error(DMRG_E_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    }
    c->stream = c->own_stream;
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    e = cudaMalloc(&c->d_status, sizeof(int) * 16);
    if (e != cudaSuccess) {
        cudaStreamDestroy(c->own_stream);
        delete c;
        return set_error(DMRG_E_NOMEM, "cudaMalloc status: %s", cudaGetErrorString(e));
    }
    cudaMemset(c->d_status, 0, sizeof(int) * 16);
    e = cudaMallocHost(&c->h_pinned, sizeof(int) * 64);
    if (e != cudaSuccess) {
        cudaFree(c->d_status);
        cudaStreamDestroy(c->own_stream);
        delete c;
        return set_error(DMRG_E_NOMEM, "cudaMallocHost: %s", cudaGetErrorString(e));
    }
    *out = c;
    return DMRG_OK;
}

int dmrg_ctx_destroy(dmrg_ctx_t ctx) {
    if (!ctx) return DMRG_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->d_status);
    cudaFreeHost(ctx->h_pinned);
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return DMRG_OK;
}

int dmrg_ctx_set_stream(dmrg_ctx_t ctx, void* stream) {
    if (!ctx) return set_error(DMRG_E_ARG, "null context");
    ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
    return DMRG_OK;
}

void* dmrg_ctx_stream(dmrg_ctx_t ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int dmrg_ctx_sync(dmrg_ctx_t ctx) {
    if (!ctx) return set_error(DMRG_E_ARG, "null context");
    DMRG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return dmrg::take_device_status(ctx);
}

int dmrg_malloc(dmrg_ctx_t ctx, size_t bytes, void** dev) {
    if (!ctx || !dev) return set_error(DMRG_E_ARG, "null argument");
    cudaError_t e = cudaMalloc(dev, bytes ? bytes : 1);
    if (e != cudaSuccess) return set_error(DMRG_E_NOMEM, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    return DMRG_OK;
}

int dmrg_free(dmrg_ctx_t ctx, void* dev) {
    (void)ctx;
    if (dev) DMRG_CUDA_TRY(cudaFree(dev));
    return DMRG_OK;
}

int dmrg_memcpy_h2d(dmrg_ctx_t ctx, void* dst, const void* src, size_t bytes) {
    if (!ctx) return set_error(DMRG_E_ARG, "null context");
    if (bytes == 0) return DMRG_OK;
    DMRG_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    DMRG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return DMRG_OK;
}

int dmrg_memcpy_d2h(dmrg_ctx_t ctx, void* dst, const void* src, size_t bytes) {
    if (!ctx) return set_error(DMRG_E_ARG, "null context");
    if (bytes == 0) return DMRG_OK;
    DMRG_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    DMRG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return DMRG_OK;
}

int dmrg_memset(dmrg_ctx_t ctx, void* dev, int value, size_t bytes) {
    if (!ctx) return set_error(DMRG_E_ARG, "null context");
    if (bytes == 0) return DMRG_OK;
    DMRG_CUDA_TRY(cudaMemsetAsync(dev, value, bytes, ctx->stream));
    return DMRG_OK;
}

}  // extern "C"
