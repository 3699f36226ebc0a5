// Small device utilities exposed through the C ABI.
#include <atomic>

#include "common.cuh"

namespace dmrg {

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

namespace {

// splitmix64 (Steele, Lea, Flood 2014) mapped to [-1, 1): element i of the stream
// seeded with `seed` is f(seed + (i + 1) * golden_gamma).
__global__ void fill_splitmix_kernel(double* __restrict__ out, int64_t n, uint64_t seed, int64_t start) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint64_t z = seed + (uint64_t)(start + i + 1) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z = z ^ (z >> 31);
        out[i] = (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
    }
}

}  // namespace
}  // namespace dmrg

using namespace dmrg;

extern "C" int dmrg_fill_uniform(dmrg_ctx_t ctx, double* dev, int64_t n, uint64_t seed, int64_t start) {
    if (!ctx || (!dev && n > 0) || n < 0) return set_error(DMRG_E_ARG, "invalid fill arguments");
    if (n == 0) return DMRG_OK;
    int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)ctx->num_sms * 8);
    DMRG_LAUNCH fill_splitmix_kernel<<<blocks, 256, 0, ctx->stream>>>(dev, n, seed, start);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

extern "C" int dmrg_launch_count(int64_t* count) {
    if (!count) return set_error(DMRG_E_ARG, "null argument");
    *count = (int64_t)g_launches.load(std::memory_order_relaxed);
    return DMRG_OK;
}
