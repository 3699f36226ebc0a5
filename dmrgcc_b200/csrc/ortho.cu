// Orthonormal kept columns from the batched Jacobi SVD (see ortho.cuh).
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "ortho.cuh"

namespace dmrg {
namespace {

// K0 of every task: column j = sign_j W[:, perm_j] / s_j (0 where s_j = 0).
// Grid (tasks, column groups of 8), one warp per column.
__global__ void __launch_bounds__(256) kform_kernel(const OrthoTask* __restrict__ tasks,
                                                    const SvdProblem* __restrict__ probs, const double* __restrict__ W,
                                                    const double* __restrict__ sig, const int* __restrict__ perm,
                                                    const double* __restrict__ sgn, double* __restrict__ K) {
    const OrthoTask t = tasks[blockIdx.x];
    const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (j >= t.t) return;
    const SvdProblem p = probs[t.problem];
    const double s = sig[p.s_off + j];
    const double f = s > 0.0 ? sgn[p.s_off + j] / s : 0.0;
    const double* w = W + p.w_off + (int64_t)perm[p.perm_off + j] * p.rows;
    double* k = K + t.k_off + (int64_t)j * t.r;
    for (int i = threadIdx.x & 31; i < t.r; i += 32) k[i] = f * w[i];
}

// G (t x t, row-major, symmetric) <- its strictly lower part.
__global__ void __launch_bounds__(256) strict_lower_kernel(const OrthoTask* __restrict__ tasks, double* __restrict__ G) {
    const OrthoTask t = tasks[blockIdx.x];
    double* g = G + t.g_off;
    for (int64_t e = threadIdx.x; e < (int64_t)t.t * t.t; e += blockDim.x)
        if (e % t.t >= e / t.t) g[e] = 0.0;
}

// Every nonzero column of K scaled to unit norm.  Grid (tasks, column groups of
// 8), one warp per column (fixed reduction order).
__global__ void __launch_bounds__(256) normalize_kernel(const OrthoTask* __restrict__ tasks, double* __restrict__ K) {
    const OrthoTask t = tasks[blockIdx.x];
    const int j = blockIdx.y * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (j >= t.t) return;
    double* k = K + t.k_off + (int64_t)j * t.r;
    double s = 0.0;
    for (int i = lane; i < t.r; i += 32) s += k[i] * k[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (s <= 0.0) return;
    const double f = 1.0 / sqrt(s);
    for (int i = lane; i < t.r; i += 32) k[i] *= f;
}

}  // namespace

int KetOrtho::plan(const BatchedSvd& svd, const std::vector<int>& kept, const std::vector<std::vector<double>>& sv,
                   cudaStream_t st, int num_sms) {
    tasks.clear();
    koff.assign(svd.probs.size(), -1);
    ksize = gsize = 0;
    cols = passes = 0;
    for (int i = 0; i < (int)svd.probs.size() && i < (int)kept.size(); ++i) {
        const int t = kept[i];
        if (t <= 0) continue;
        const SvdProblem& p = svd.probs[i];
        if (t > p.cols) return set_error(DMRG_E_ARG, "orthonormalisation of %d columns of a %d-column factor", t, p.cols);
        // the sweeps leave |u_a . u_b| <= tol ||A||_F / min(s_a, s_b)
        double fro2 = 0.0;
        for (double v : sv[i]) fro2 += v * v;
        const double smin = t - 1 < (int)sv[i].size() ? sv[i][t - 1] : 0.0;
        const double tol = 2.0 * DBL_EPSILON * std::sqrt((double)p.rows);
        const double e = smin > 0.0 ? tol * std::sqrt(fro2) / smin : 1.0;
        int n = 1;
        for (double x = e; x > 1e-16 && n < 6; x *= x) ++n;
        if (e >= 0.5) n = 6;
        passes = std::max(passes, n);
        koff[i] = ksize;
        tasks.push_back(OrthoTask{i, t, p.rows, 0, ksize, gsize});
        cols = std::max(cols, t);
        ksize += (int64_t)p.rows * t;
        gsize += (int64_t)t * t;
    }
    if (tasks.empty()) return DMRG_OK;
    DMRG_TRY(d_k.alloc(ksize * sizeof(double)));
    DMRG_TRY(d_k2.alloc(ksize * sizeof(double)));
    DMRG_TRY(d_g.alloc(gsize * sizeof(double)));
    DMRG_TRY(upload(d_tasks, tasks, st));
    sg.reset();
    su.reset();
    sg.tb = true;  // G = K^T K: K^T is K column-major read row-major (t x r), K the transposed B
    for (const OrthoTask& o : tasks) {
        sg.add_group(o.g_off, o.t, o.t, o.t);
        sg.add_term(o.k_off, o.r, o.k_off, o.r, o.r, 1.0);
        // K2^T (row-major t x r) -= L (t x t) K^T
        su.add_group(o.k_off, o.r, o.t, o.r);
        su.add_term(o.g_off, o.t, o.k_off, o.r, o.t, -1.0);
    }
    DMRG_TRY(sg.check_bounds(ksize, ksize, gsize));
    DMRG_TRY(su.check_bounds(gsize, ksize, ksize));
    DMRG_TRY(sg.finalize(64, 64, 16, st, num_sms));
    DMRG_TRY(su.finalize(64, 64, 16, st, num_sms));
    return DMRG_OK;
}

int KetOrtho::run(const BatchedSvd& svd, cudaStream_t st) {
    if (tasks.empty()) return DMRG_OK;
    const int nt = (int)tasks.size();
    const dim3 grid(nt, (cols + 7) / 8);
    const OrthoTask* ot = d_tasks.as<OrthoTask>();
    DMRG_LAUNCH kform_kernel<<<grid, 256, 0, st>>>(ot, svd.d_probs.as<SvdProblem>(), svd.d_w.as<double>(),
                                                   svd.d_s.as<double>(), svd.d_perm.as<int>(), svd.d_sign.as<double>(),
                                                   d_k.as<double>());
    DMRG_CUDA_TRY(cudaGetLastError());
    for (int pass = 0; pass < passes; ++pass) {
        DeviceBuffer& k = pass % 2 == 0 ? d_k : d_k2;
        DeviceBuffer& k2 = pass % 2 == 0 ? d_k2 : d_k;
        DMRG_TRY(launch_gemm_f64(sg, k.as<double>(), k.as<double>(), d_g.as<double>(), false, st));
        DMRG_LAUNCH strict_lower_kernel<<<nt, 256, 0, st>>>(ot, d_g.as<double>());
        DMRG_CUDA_TRY(cudaMemcpyAsync(k2.ptr, k.ptr, ksize * sizeof(double), cudaMemcpyDeviceToDevice, st));
        DMRG_TRY(launch_gemm_f64(su, d_g.as<double>(), k.as<double>(), k2.as<double>(), true, st));
        DMRG_LAUNCH normalize_kernel<<<grid, 256, 0, st>>>(ot, k2.as<double>());
        DMRG_CUDA_TRY(cudaGetLastError());
    }
    return DMRG_OK;
}

}  // namespace dmrg
