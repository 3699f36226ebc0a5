// FP64 throughput probe.  MEASURED_PEAKS-style figures exist for bf16 and HBM
// only, so the FP64 roofline denominator of the block GEMMs is measured here:
// a register-resident loop of independent DMMA (mma.sync m8n8k4 f64) or DFMA
// instructions on every SM, timed with CUDA events.
#include "common.cuh"

namespace dmrg {
namespace {

__global__ void __launch_bounds__(128) dmma_loop(double* sink, int iters) {
    double acc[8][2];
    double a = 1.0 + threadIdx.x * 1e-9, b = 1.0 - threadIdx.x * 1e-9;
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = 0.0;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                         : "+d"(acc[i][0]), "+d"(acc[i][1])
                         : "d"(a), "d"(b));
    }
    double s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += acc[i][0] + acc[i][1];
    if (s == 12345.678) sink[0] = s;  // never true; keeps the loop alive
}

__global__ void __launch_bounds__(256) dfma_loop(double* sink, int iters) {
    double acc[8];
    const double a = 1.0 + threadIdx.x * 1e-9, b = 1.0 - threadIdx.x * 1e-12;
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i] = i;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[i] = fma(acc[i], a, b);
    }
    double s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += acc[i];
    if (s == 12345.678) sink[0] = s;
}

}  // namespace
}  // namespace dmrg

using namespace dmrg;

// mode 0: DMMA, mode 1: DFMA.  *tflops receives the achieved FP64 TFLOP/s.
extern "C" int dmrg_fp64_peak(dmrg_ctx_t ctx, int mode, int iters, double* tflops) {
    if (!ctx || !tflops || iters <= 0 || (mode != 0 && mode != 1)) return set_error(DMRG_E_ARG, "bad arguments");
    DeviceBuffer sink;
    DMRG_TRY(sink.alloc(64));
    cudaEvent_t e0, e1;
    DMRG_CUDA_TRY(cudaEventCreate(&e0));
    DMRG_CUDA_TRY(cudaEventCreate(&e1));
    const int blocks = ctx->num_sms * 8;
    double flops;
    // warm-up
    if (mode == 0) DMRG_LAUNCH dmma_loop<<<blocks, 128, 0, ctx->stream>>>(sink.as<double>(), iters / 10 + 1);
    else DMRG_LAUNCH dfma_loop<<<blocks, 256, 0, ctx->stream>>>(sink.as<double>(), iters / 10 + 1);
    cudaEventRecord(e0, ctx->stream);
    if (mode == 0) {
        DMRG_LAUNCH dmma_loop<<<blocks, 128, 0, ctx->stream>>>(sink.as<double>(), iters);
        flops = (double)blocks * 4 /*warps*/ * iters * 8 * (8.0 * 8 * 4 * 2);
    } else {
        DMRG_LAUNCH dfma_loop<<<blocks, 256, 0, ctx->stream>>>(sink.as<double>(), iters);
        flops = (double)blocks * 256 * iters * 8 * 2.0;
    }
    cudaEventRecord(e1, ctx->stream);
    DMRG_CUDA_TRY(cudaGetLastError());
    DMRG_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *tflops = flops / (ms * 1e-3) * 1e-12;
    return DMRG_OK;
}
