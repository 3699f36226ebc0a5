// Batched one-sided block-Jacobi SVD (see svd.cuh).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "svd.cuh"

namespace dmrg {
namespace {

constexpr int kBlk = 32;        // columns per block
constexpr int kPair = 64;       // columns per pair
constexpr int kChunk = 32;      // rows per streamed chunk
constexpr int kThreads = 256;
constexpr int kLd = kPair + 1;  // padded row of the shared 64x64 matrices
constexpr int kInnerSweeps = 4;
constexpr int kMaxSweeps = 40;
// Columns whose norm is below kZeroRel * sqrt(rows) * ||A||_F are rounding
// residue of a rank-deficient matrix: they take part in no rotation and in no
// convergence test (their values are below any truncation threshold that is
// meaningful in FP64; rotating them only stirs rounding noise).
constexpr double kZeroRel = 4.0 * DBL_EPSILON;

struct SvdSmem {
    double G[kPair * kLd];
    double Q[kPair * kLd];
    double X[kChunk * kLd];
    double cs[kPair];
    int pq[kPair];
    double red[kThreads / 32];
    double flag;
};

__device__ __forceinline__ void rr_pair(int r, int i, int N, int& p, int& q) {
    if (i == 0) {
        p = 0;
        q = r % (N - 1) + 1;
    } else {
        p = (r + i) % (N - 1) + 1;
        q = (r - i + (N - 1)) % (N - 1) + 1;
    }
    if (p > q) {
        const int t = p;
        p = q;
        q = t;
    }
}

__device__ double block_max(double v, SvdSmem& S) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) S.red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) m = fmax(m, S.red[w]);
        S.flag = m;
    }
    __syncthreads();
    const double r = S.flag;
    __syncthreads();
    return r;
}

// Loads rows [k0, k0+kChunk) of the pair's 64 columns (zero outside) into S.X[k][c].
__device__ __forceinline__ void load_chunk(SvdSmem& S, const double* __restrict__ base, int ld, int nrows,
                                           int ncols, int colI, int colJ, int k0) {
    for (int idx = threadIdx.x; idx < kChunk * kPair; idx += kThreads) {
        const int c = idx / kChunk, k = idx % kChunk;
        const int gc = c < kBlk ? colI + c : colJ + c - kBlk;
        const bool v = gc < ncols && k0 + k < nrows;
        S.X[k * kLd + c] = v ? base[(int64_t)gc * ld + k0 + k] : 0.0;
    }
}

__device__ __forceinline__ void store_chunk(SvdSmem& S, double* __restrict__ base, int ld, int nrows, int ncols,
                                            int colI, int colJ, int k0) {
    for (int idx = threadIdx.x; idx < kChunk * kPair; idx += kThreads) {
        const int c = idx / kChunk, k = idx % kChunk;
        const int gc = c < kBlk ? colI + c : colJ + c - kBlk;
        if (gc < ncols && k0 + k < nrows) base[(int64_t)gc * ld + k0 + k] = S.X[k * kLd + c];
    }
}

// X (kChunk x 64, in S.X) <- X * Q  (in place through registers)
__device__ __forceinline__ void rotate_chunk(SvdSmem& S) {
    const int k = threadIdx.x / 8, c0 = (threadIdx.x % 8) * 8;
    double y[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) y[e] = 0.0;
    for (int c = 0; c < kPair; ++c) {
        const double x = S.X[k * kLd + c];
#pragma unroll
        for (int e = 0; e < 8; ++e) y[e] += x * S.Q[c * kLd + c0 + e];
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < 8; ++e) S.X[k * kLd + c0 + e] = y[e];
    __syncthreads();
}

__global__ void __launch_bounds__(kThreads) jacobi_round_kernel(const SvdProblem* __restrict__ probs,
                                                                const SvdTask* __restrict__ tasks, int round,
                                                                double* __restrict__ W, double* __restrict__ Qacc,
                                                                const double* __restrict__ fro2,
                                                                unsigned long long* __restrict__ conv) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SvdSmem& S = *reinterpret_cast<SvdSmem*>(smem_raw);
    const SvdTask task = tasks[blockIdx.x];
    const SvdProblem p = probs[task.problem];
    int I, J;
    rr_pair(round, task.pair, p.nbe, I, J);
    const int colI = I * kBlk, colJ = J * kBlk;
    double* Wp = W + p.w_off;
    double* Qp = Qacc + p.q_off;
    const double tol = 2.0 * DBL_EPSILON * sqrt((double)p.rows);
    const double zero2 = kZeroRel * kZeroRel * (double)p.rows * fro2[task.problem];

    // ---- Gram matrix of the pair: G = X^T X over all rows -----------------------
    const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;  // 4x4 micro-tile (rows ty*4.., cols tx*4..)
    double g[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) g[a][b] = 0.0;
    for (int k0 = 0; k0 < p.rows; k0 += kChunk) {
        load_chunk(S, Wp, p.rows, p.rows, p.cols, colI, colJ, k0);
        __syncthreads();
        for (int k = 0; k < kChunk; ++k) {
            double xa[4], xb[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) xa[a] = S.X[k * kLd + ty * 4 + a];
#pragma unroll
            for (int b = 0; b < 4; ++b) xb[b] = S.X[k * kLd + tx * 4 + b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) g[a][b] += xa[a] * xb[b];
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) S.G[(ty * 4 + a) * kLd + tx * 4 + b] = g[a][b];
    for (int idx = threadIdx.x; idx < kPair * kPair; idx += kThreads)
        S.Q[(idx / kPair) * kLd + idx % kPair] = (idx / kPair == idx % kPair) ? 1.0 : 0.0;
    __syncthreads();

    // ---- outer convergence measure: max |g_ij| / sqrt(g_ii g_jj) over the pair --
    double worst = 0.0;
    for (int idx = threadIdx.x; idx < kPair * kPair; idx += kThreads) {
        const int a = idx / kPair, b = idx % kPair;
        if (a >= b) continue;
        const double ga = S.G[a * kLd + a], gb = S.G[b * kLd + b];
        if (ga > zero2 && gb > zero2) worst = fmax(worst, fabs(S.G[a * kLd + b]) / sqrt(ga * gb));
    }
    worst = block_max(worst, S);
    if (threadIdx.x == 0) atomicMax(conv + task.problem, (unsigned long long)__double_as_longlong(worst));
    if (worst <= tol) return;  // pair already orthogonal: nothing to rotate

    // ---- inner cyclic Jacobi on the 64x64 Gram matrix, accumulating Q ----------
    for (int sweep = 0; sweep < kInnerSweeps; ++sweep) {
        for (int r = 0; r < kPair - 1; ++r) {
            if (threadIdx.x < kPair / 2) {
                int a, b;
                rr_pair(r, threadIdx.x, kPair, a, b);
                const double apq = S.G[a * kLd + b];
                double c = 1.0, s = 0.0;
                const double daa = S.G[a * kLd + a], dbb = S.G[b * kLd + b];
                if (apq != 0.0 && daa > zero2 && dbb > zero2 && fabs(apq) > DBL_EPSILON * 1e-3 * sqrt(daa * dbb)) {
                    const double tau = (dbb - daa) / (2.0 * apq);
                    const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                    c = 1.0 / sqrt(1.0 + t * t);
                    s = t * c;
                }
                S.cs[2 * threadIdx.x] = c;
                S.cs[2 * threadIdx.x + 1] = s;
                S.pq[2 * threadIdx.x] = a;
                S.pq[2 * threadIdx.x + 1] = b;
            }
            __syncthreads();
            for (int idx = threadIdx.x; idx < (kPair / 2) * kPair; idx += kThreads) {
                const int i = idx / kPair, j = idx % kPair;
                const double s = S.cs[2 * i + 1];
                if (s == 0.0) continue;
                const double c = S.cs[2 * i];
                const int a = S.pq[2 * i], b = S.pq[2 * i + 1];
                const double ga = S.G[a * kLd + j], gb = S.G[b * kLd + j];
                S.G[a * kLd + j] = c * ga - s * gb;
                S.G[b * kLd + j] = s * ga + c * gb;
            }
            __syncthreads();
            for (int idx = threadIdx.x; idx < (kPair / 2) * kPair; idx += kThreads) {
                const int i = idx / kPair, row = idx % kPair;
                const double s = S.cs[2 * i + 1];
                if (s == 0.0) continue;
                const double c = S.cs[2 * i];
                const int a = S.pq[2 * i], b = S.pq[2 * i + 1];
                const double ga = S.G[row * kLd + a], gb = S.G[row * kLd + b];
                S.G[row * kLd + a] = c * ga - s * gb;
                S.G[row * kLd + b] = s * ga + c * gb;
                const double qa = S.Q[row * kLd + a], qb = S.Q[row * kLd + b];
                S.Q[row * kLd + a] = c * qa - s * qb;
                S.Q[row * kLd + b] = s * qa + c * qb;
            }
            __syncthreads();
        }
    }

    // ---- apply the pair rotation to W's and to the accumulated rotation's columns
    for (int k0 = 0; k0 < p.rows; k0 += kChunk) {
        load_chunk(S, Wp, p.rows, p.rows, p.cols, colI, colJ, k0);
        __syncthreads();
        rotate_chunk(S);
        store_chunk(S, Wp, p.rows, p.rows, p.cols, colI, colJ, k0);
        __syncthreads();
    }
    for (int k0 = 0; k0 < p.cols; k0 += kChunk) {
        load_chunk(S, Qp, p.cols, p.cols, p.cols, colI, colJ, k0);
        __syncthreads();
        rotate_chunk(S);
        store_chunk(S, Qp, p.cols, p.cols, p.cols, colI, colJ, k0);
        __syncthreads();
    }
}

// Squared Frobenius norm of each working matrix (fixed-order block reduction).
__global__ void __launch_bounds__(256) fro2_kernel(const SvdProblem* __restrict__ probs, const double* __restrict__ W,
                                                   double* __restrict__ fro2) {
    __shared__ double red[256];
    const SvdProblem p = probs[blockIdx.x];
    const double* w = W + p.w_off;
    double s = 0.0;
    for (int64_t i = threadIdx.x; i < (int64_t)p.rows * p.cols; i += blockDim.x) s += w[i] * w[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) fro2[blockIdx.x] = red[0];
}

__global__ void init_identity_kernel(const SvdProblem* __restrict__ probs, double* __restrict__ Q) {
    const SvdProblem p = probs[blockIdx.x];
    double* q = Q + p.q_off;
    for (int64_t idx = threadIdx.x; idx < (int64_t)p.cols * p.cols; idx += blockDim.x)
        q[idx] = (idx / p.cols == idx % p.cols) ? 1.0 : 0.0;
}

// Column norms -> singular values, sorted descending (ties by column index).
__global__ void __launch_bounds__(256) finalize_kernel(const SvdProblem* __restrict__ probs,
                                                       const double* __restrict__ W, double* __restrict__ sig,
                                                       int* __restrict__ perm, double* __restrict__ tmp) {
    const SvdProblem p = probs[blockIdx.x];
    const double* Wp = W + p.w_off;
    double* t = tmp + p.s_off;
    for (int j = threadIdx.x; j < p.cols; j += blockDim.x) {
        const double* col = Wp + (int64_t)j * p.rows;
        double s = 0.0;
        for (int k = 0; k < p.rows; ++k) s += col[k] * col[k];
        t[j] = sqrt(s);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < p.cols; j += blockDim.x) {
        const double v = t[j];
        int rank = 0;
        for (int o = 0; o < p.cols; ++o) {
            const double u = t[o];
            rank += (u > v) || (u == v && o < j);
        }
        sig[p.s_off + rank] = v;
        perm[p.perm_off + rank] = j;
    }
}

// Sign convention for each singular triplet (rank j, sorted): the left singular
// vector u_j is taken with its largest-magnitude component positive; components
// within a relative 1e-6 of the largest count as equal and the first decides.
// u_j is column perm[j] of W (scaled by 1/s_j) when W = A, of Q when W = A^T.
// One warp per rank.
__global__ void __launch_bounds__(256) sign_kernel(const SvdProblem* __restrict__ probs, const double* __restrict__ W,
                                                   const double* __restrict__ Q, const int* __restrict__ perm,
                                                   double* __restrict__ sign) {
    const SvdProblem p = probs[blockIdx.x];
    const int lane = threadIdx.x & 31;
    const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (j >= p.cols) return;
    const int k = perm[p.perm_off + j];
    const double* u = p.transposed ? Q + p.q_off + (int64_t)k * p.m : W + p.w_off + (int64_t)k * p.m;
    double mx = 0.0;
    for (int i = lane; i < p.m; i += 32) mx = fmax(mx, fabs(u[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    int first = p.m;
    for (int i = lane; i < p.m; i += 32)
        if (mx > 0.0 && fabs(u[i]) >= mx * (1.0 - 1e-6)) {
            first = i;
            break;
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) first = min(first, __shfl_xor_sync(0xffffffffu, first, o));
    if (lane == 0) sign[p.s_off + j] = (first < p.m && u[first] < 0.0) ? -1.0 : 1.0;
}

}  // namespace

int BatchedSvd::plan(const std::vector<int>& m, const std::vector<int>& n, cudaStream_t st) {
    probs.clear();
    tasks.clear();
    round_first.clear();
    index.assign(m.size(), -1);
    int64_t woff = 0, qoff = 0, soff = 0;
    max_rounds = 0;
    for (size_t i = 0; i < m.size(); ++i) {
        if ((int64_t)m[i] * n[i] <= 0) continue;
        SvdProblem p{};
        p.m = m[i];
        p.n = n[i];
        p.transposed = n[i] > m[i];
        p.rows = p.transposed ? n[i] : m[i];
        p.cols = p.transposed ? m[i] : n[i];
        const int nb = (p.cols + kBlk - 1) / kBlk;
        p.nbe = std::max(2, nb + (nb & 1));
        p.w_off = woff;
        p.q_off = qoff;
        p.s_off = soff;
        p.perm_off = soff;
        woff += (int64_t)p.rows * p.cols;
        qoff += (int64_t)p.cols * p.cols;
        soff += p.cols;
        index[i] = (int)probs.size();
        probs.push_back(p);
        max_rounds = std::max(max_rounds, p.nbe - 1);
    }
    for (int r = 0; r < max_rounds; ++r) {
        round_first.push_back((int)tasks.size());
        for (int pi = 0; pi < (int)probs.size(); ++pi)
            if (r < probs[pi].nbe - 1)
                for (int k = 0; k < probs[pi].nbe / 2; ++k) tasks.push_back(SvdTask{pi, k});
    }
    round_first.push_back((int)tasks.size());
    DMRG_TRY(d_w.alloc((size_t)std::max<int64_t>(woff, 1) * sizeof(double)));
    DMRG_TRY(d_q.alloc((size_t)std::max<int64_t>(qoff, 1) * sizeof(double)));
    DMRG_TRY(d_s.alloc((size_t)std::max<int64_t>(2 * soff, 1) * sizeof(double)));
    DMRG_TRY(d_perm.alloc((size_t)std::max<int64_t>(soff, 1) * sizeof(int)));
    DMRG_TRY(d_conv.alloc(std::max<size_t>(probs.size(), 1) * sizeof(unsigned long long)));
    DMRG_TRY(d_fro2.alloc(std::max<size_t>(probs.size(), 1) * sizeof(double)));
    DMRG_TRY(d_sign.alloc((size_t)std::max<int64_t>(soff, 1) * sizeof(double)));
    DMRG_TRY(upload(d_probs, probs, st));
    DMRG_TRY(upload(d_tasks, tasks, st));
    DMRG_CUDA_TRY(cudaFuncSetAttribute(jacobi_round_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(SvdSmem)));
    return DMRG_OK;
}

int BatchedSvd::run(cudaStream_t st, int* sweeps_out) {
    if (probs.empty()) {
        if (sweeps_out) *sweeps_out = 0;
        return DMRG_OK;
    }
    const int np = (int)probs.size();
    init_identity_kernel<<<np, 256, 0, st>>>(d_probs.as<SvdProblem>(), d_q.as<double>());
    fro2_kernel<<<np, 256, 0, st>>>(d_probs.as<SvdProblem>(), d_w.as<double>(), d_fro2.as<double>());
    std::vector<unsigned long long> conv(np);
    int sweep = 0, worst_at = 0;
    double worst_left = 0.0;
    for (; sweep < kMaxSweeps; ++sweep) {
        DMRG_CUDA_TRY(cudaMemsetAsync(d_conv.ptr, 0, np * sizeof(unsigned long long), st));
        for (int r = 0; r < max_rounds; ++r) {
            const int n = round_first[r + 1] - round_first[r];
            if (n == 0) continue;
            jacobi_round_kernel<<<n, kThreads, sizeof(SvdSmem), st>>>(
                d_probs.as<SvdProblem>(), d_tasks.as<SvdTask>() + round_first[r], r, d_w.as<double>(),
                d_q.as<double>(), d_fro2.as<double>(), d_conv.as<unsigned long long>());
        }
        DMRG_CUDA_TRY(cudaGetLastError());
        DMRG_CUDA_TRY(cudaMemcpyAsync(conv.data(), d_conv.ptr, np * sizeof(unsigned long long),
                                      cudaMemcpyDeviceToHost, st));
        DMRG_CUDA_TRY(cudaStreamSynchronize(st));
        bool done = true;
        for (int i = 0; i < np; ++i) {
            double worst;
            std::memcpy(&worst, &conv[i], sizeof(double));
            if (worst > 2.0 * DBL_EPSILON * std::sqrt((double)probs[i].rows)) {
                done = false;
                if (sweep == kMaxSweeps - 1 && worst > worst_left) {
                    worst_left = worst;
                    worst_at = i;
                }
            }
        }
        if (done) break;
    }
    if (sweep == kMaxSweeps)
        return set_error(DMRG_E_NUMERIC, "Jacobi SVD did not converge in %d sweeps (sector %d x %d: off-diagonal %.3e)",
                         kMaxSweeps, probs[worst_at].m, probs[worst_at].n, worst_left);
    finalize_kernel<<<np, 256, 0, st>>>(d_probs.as<SvdProblem>(), d_w.as<double>(), d_s.as<double>(),
                                        d_perm.as<int>(), d_s.as<double>() + (d_s.bytes / sizeof(double)) / 2);
    int max_cols = 0;
    for (const SvdProblem& p : probs) max_cols = std::max(max_cols, p.cols);
    sign_kernel<<<dim3(np, (max_cols + 7) / 8), 256, 0, st>>>(d_probs.as<SvdProblem>(), d_w.as<double>(),
                                                               d_q.as<double>(), d_perm.as<int>(), d_sign.as<double>());
    DMRG_CUDA_TRY(cudaGetLastError());
    if (sweeps_out) *sweeps_out = sweep + 1;
    return DMRG_OK;
}

int BatchedSvd::singular_values(std::vector<std::vector<double>>& out, cudaStream_t st) {
    out.assign(index.size(), std::vector<double>());
    if (probs.empty()) return DMRG_OK;
    int64_t total = 0;
    for (const auto& p : probs) total += p.cols;
    std::vector<double> all(total);
    DMRG_CUDA_TRY(cudaMemcpyAsync(all.data(), d_s.ptr, total * sizeof(double), cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaStreamSynchronize(st));
    for (size_t i = 0; i < index.size(); ++i) {
        if (index[i] < 0) continue;
        const SvdProblem& p = probs[index[i]];
        out[i].assign(all.begin() + p.s_off, all.begin() + p.s_off + p.cols);
    }
    return DMRG_OK;
}

}  // namespace dmrg
