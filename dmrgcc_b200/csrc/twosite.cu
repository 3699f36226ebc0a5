// Two-site split kernels (see twosite.cuh).  HBM-bound block copies: one CTA
// per block, coalesced over the block's row-major elements.
#include <algorithm>
#include <tuple>

#include "twosite.cuh"

namespace dmrg {
namespace {

// Theta block -> its place in the sector's working matrix W (column-major;
// W = M_c, or W = M_c^T when the batch transposed it).
__global__ void twosite_gather_kernel(const double* __restrict__ theta, const SplitBlock* __restrict__ blocks,
                                      const int* __restrict__ batch, const SvdProblem* __restrict__ probs,
                                      double* __restrict__ W) {
    const SplitBlock b = blocks[blockIdx.x];
    const SvdProblem p = probs[batch[b.sector]];
    const double* src = theta + b.theta_off;
    double* w = W + p.w_off;
    const int64_t total = (int64_t)b.rows * b.cols;
    for (int64_t e = threadIdx.x; e < total; e += blockDim.x) {
        const int ai = b.row0 + (int)(e / b.cols), aj = b.col0 + (int)(e % b.cols);
        if (ai >= p.m || aj >= p.n) continue;
        w[p.transposed ? (int64_t)ai * p.n + aj : (int64_t)aj * p.m + ai] = src[e];
    }
}

// New site-tensor blocks from the batch's factors.  After the Jacobi sweeps a
// plain batch (W = M) holds the columns u_k s_k in W and V in Q; a transposed
// one (W = M^T) holds v_k s_k in W and U in Q; perm orders by descending s and
// sgn fixes each pair's sign.
__global__ void twosite_write_kernel(const SplitWrite* __restrict__ writes, const int* __restrict__ batch,
                                     const SvdProblem* __restrict__ probs, const double* __restrict__ W,
                                     const double* __restrict__ Q, const double* __restrict__ sig,
                                     const int* __restrict__ perm, const double* __restrict__ sgn,
                                     double* __restrict__ left, double* __restrict__ right, int s_left,
                                     const double* __restrict__ K, const double* __restrict__ P) {
    const SplitWrite t = writes[blockIdx.x];
    const SvdProblem p = probs[batch[t.sector]];
    const double* w = W + p.w_off;
    const double* q = Q + p.q_off;
    double* out = t.part == 0 ? left : right;
    const int64_t total = (int64_t)t.rows * t.cols;
    if (t.k_off >= 0) {  // orthonormalised columns: U[row][j] (part 0) or V^T[i][col] (part 1)
        const double* k = K + t.k_off;
        for (int64_t e = threadIdx.x; e < total; e += blockDim.x) {
            const int i = (int)(e / t.cols), j = (int)(e % t.cols);
            out[t.out_off + e] = t.part == 0 ? k[(int64_t)j * p.rows + t.off + i] : k[(int64_t)i * p.rows + t.off + j];
        }
        return;
    }
    if (t.p_off >= 0) {  // projected factor: S V^T columns (part 1, t x n) or U S rows (part 0, m x t)
        const double* pr = P + t.p_off;
        for (int64_t e = threadIdx.x; e < total; e += blockDim.x) {
            const int i = (int)(e / t.cols), j = (int)(e % t.cols);
            out[t.out_off + e] = t.part == 1 ? pr[(int64_t)i * p.n + t.off + j] : pr[(int64_t)(t.off + i) * t.cols + j];
        }
        return;
    }
    for (int64_t e = threadIdx.x; e < total; e += blockDim.x) {
        const int i = (int)(e / t.cols), j = (int)(e % t.cols);
        double v;
        if (t.part == 0) {  // U[row][j] (times s_j when s_left)
            const int k = perm[p.perm_off + j];
            const int row = t.off + i;
            const double s = sig[p.s_off + j];
            if (!p.transposed) {
                const double us = w[(int64_t)k * p.m + row];
                v = s_left ? us : (s > 0.0 ? us / s : 0.0);
            } else {
                const double u = q[(int64_t)k * p.m + row];
                v = s_left ? u * s : u;
            }
            v *= sgn[p.s_off + j];
        } else {  // V^T[i][col] (times s_i unless s_left)
            const int k = perm[p.perm_off + i];
            const int col = t.off + j;
            const double s = sig[p.s_off + i];
            if (!p.transposed) {
                const double vv = q[(int64_t)k * p.n + col];
                v = s_left ? vv : vv * s;
            } else {
                const double vs = w[(int64_t)k * p.n + col];
                v = s_left ? (s > 0.0 ? vs / s : 0.0) : vs;
            }
            v *= sgn[p.s_off + i];
        }
        out[t.out_off + e] = v;
    }
}

}  // namespace

int twosite_gather(BatchedSvd& svd, const std::vector<int>& sector_batch, const double* theta,
                   const std::vector<SplitBlock>& blocks, DeviceBuffer& d_blocks, cudaStream_t st, double* dst) {
    int64_t wsize = 0;
    for (const auto& p : svd.probs) wsize += (int64_t)p.rows * p.cols;
    double* W = dst ? dst : svd.d_w.as<double>();
    if (wsize) DMRG_CUDA_TRY(cudaMemsetAsync(W, 0, wsize * sizeof(double), st));
    std::vector<SplitBlock> active;
    for (const SplitBlock& b : blocks)
        if (sector_batch[b.sector] >= 0 && b.rows > 0 && b.cols > 0) active.push_back(b);
    if (active.empty()) return DMRG_OK;
    for (const SplitBlock& b : active) {
        const SvdProblem& p = svd.probs[sector_batch[b.sector]];
        if (b.row0 < 0 || b.col0 < 0 || b.row0 + b.rows > p.m || b.col0 + b.cols > p.n)
            return set_error(DMRG_E_ARG, "two-site block outside its sector matrix");
    }
    DeviceBuffer d_batch;
    DMRG_TRY(upload(d_batch, sector_batch, st));
    DMRG_TRY(upload(d_blocks, active, st));
    DMRG_LAUNCH twosite_gather_kernel<<<(int)active.size(), 256, 0, st>>>(
        theta, d_blocks.as<SplitBlock>(), d_batch.as<int>(), svd.d_probs.as<SvdProblem>(), W);
    DMRG_CUDA_TRY(cudaGetLastError());
    DMRG_CUDA_TRY(cudaStreamSynchronize(st));  // d_batch is released on return
    return DMRG_OK;
}

int twosite_write(BatchedSvd& svd, const std::vector<int>& sector_batch, const std::vector<SplitWrite>& writes,
                  DeviceBuffer& d_writes, double* left, double* right, bool s_left, cudaStream_t st,
                  const double* K, const double* P) {
    std::vector<SplitWrite> active;
    for (const SplitWrite& t : writes)
        if (t.rows > 0 && t.cols > 0) {
            if (sector_batch[t.sector] < 0) return set_error(DMRG_E_ARG, "two-site write from an empty sector");
            const SvdProblem& p = svd.probs[sector_batch[t.sector]];
            const int kept = t.part == 0 ? t.cols : t.rows;
            const int span = t.part == 0 ? t.off + t.rows : t.off + t.cols;
            if (kept > std::min(p.m, p.n) || span > (t.part == 0 ? p.m : p.n))
                return set_error(DMRG_E_ARG, "two-site write outside its sector's factors");
            if ((t.k_off >= 0 && !K) || (t.p_off >= 0 && !P))
                return set_error(DMRG_E_ARG, "two-site write from a missing orthonormalised factor");
            active.push_back(t);
        }
    if (active.empty()) return DMRG_OK;
    DeviceBuffer d_batch;
    DMRG_TRY(upload(d_batch, sector_batch, st));
    DMRG_TRY(upload(d_writes, active, st));
    DMRG_LAUNCH twosite_write_kernel<<<(int)active.size(), 256, 0, st>>>(
        d_writes.as<SplitWrite>(), d_batch.as<int>(), svd.d_probs.as<SvdProblem>(), svd.d_w.as<double>(),
        svd.d_q.as<double>(), svd.d_s.as<double>(), svd.d_perm.as<int>(), svd.d_sign.as<double>(), left, right,
        s_left ? 1 : 0, K, P);
    DMRG_CUDA_TRY(cudaGetLastError());
    DMRG_CUDA_TRY(cudaStreamSynchronize(st));
    return DMRG_OK;
}

std::vector<int> truncate_twosite(int max_dim, double canpre, const std::vector<std::vector<double>>& svals) {
    std::vector<int> tdim(svals.size(), 0);
    std::vector<std::tuple<double, int, int>> all;  // value, sector, position
    for (int s = 0; s < (int)svals.size(); ++s)
        for (int i = 0; i < (int)svals[s].size(); ++i)
            if (svals[s][i] > canpre) all.emplace_back(svals[s][i], s, i);
    if (max_dim > 0 && (int)all.size() > max_dim) {
        std::stable_sort(all.begin(), all.end(), [](const auto& a, const auto& b) {
            if (std::get<0>(a) != std::get<0>(b)) return std::get<0>(a) > std::get<0>(b);
            if (std::get<1>(a) != std::get<1>(b)) return std::get<1>(a) < std::get<1>(b);
            return std::get<2>(a) < std::get<2>(b);
        });
        all.resize(max_dim);
    }
    for (const auto& t : all) ++tdim[std::get<1>(t)];
    return tdim;
}

}  // namespace dmrg
