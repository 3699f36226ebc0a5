// Block-list data movement kernels (see blockops.cuh).  Copies are HBM-bound:
// one CTA per rectangle, rows handled by warps, consecutive threads on
// consecutive columns (coalesced on both sides).
#include "blockops.cuh"

namespace dmrg {
namespace {

__global__ void __launch_bounds__(256) rect_copy_kernel(const RectCopy* __restrict__ tasks,
                                                        const double* __restrict__ src, double* __restrict__ dst) {
    const RectCopy t = tasks[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = warp; i < t.rows; i += blockDim.x >> 5) {
        const double* s = src + t.src_off + (int64_t)i * t.src_ld;
        double* d = dst + t.dst_off + (int64_t)i * t.dst_ld;
        for (int j = lane; j < t.cols; j += 32) d[j] = t.scale * s[j];
    }
}

__global__ void scale_by_kernel(double* __restrict__ x, int64_t n, const double* __restrict__ s, int inverse) {
    const double f = inverse ? 1.0 / *s : *s;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] *= f;
}

}  // namespace

int launch_rect_copies(const std::vector<RectCopy>& tasks, const double* src, int64_t src_size, double* dst,
                       int64_t dst_size, DeviceBuffer& scratch, cudaStream_t st) {
    if (tasks.empty()) return DMRG_OK;
    for (const RectCopy& t : tasks) {
        if (t.rows <= 0 || t.cols <= 0) continue;
        const int64_t se = t.src_off + (int64_t)(t.rows - 1) * t.src_ld + t.cols;
        const int64_t de = t.dst_off + (int64_t)(t.rows - 1) * t.dst_ld + t.cols;
        if (t.src_off < 0 || t.dst_off < 0 || se > src_size || de > dst_size || t.cols > t.src_ld || t.cols > t.dst_ld)
            return set_error(DMRG_E_ARG, "block copy outside its buffers (src end %lld of %lld, dst end %lld of %lld)",
                             (long long)se, (long long)src_size, (long long)de, (long long)dst_size);
    }
    DMRG_TRY(scratch.alloc(tasks.size() * sizeof(RectCopy)));
    DMRG_CUDA_TRY(cudaMemcpyAsync(scratch.ptr, tasks.data(), tasks.size() * sizeof(RectCopy), cudaMemcpyHostToDevice,
                                  st));
    DMRG_LAUNCH rect_copy_kernel<<<(int)tasks.size(), 256, 0, st>>>(scratch.as<RectCopy>(), src, dst);
    // (a pageable-source cudaMemcpyAsync returns once the source is staged, so the
    // host vector may go away; `scratch` must outlive the launch)
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int launch_scale_by(double* x, int64_t n, const double* s, bool inverse, cudaStream_t st) {
    if (n <= 0) return DMRG_OK;
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, 1184);
    DMRG_LAUNCH scale_by_kernel<<<blocks, 256, 0, st>>>(x, n, s, inverse ? 1 : 0);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

}  // namespace dmrg
