// FP64 vector kernels (see vec.cuh).  These are HBM-bound: each reads its
// operands once with coalesced grid-stride loops and reduces deterministically.
#include "vec.cuh"

namespace dmrg {
namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the block; result valid in thread 0.
__device__ double block_sum(double v) {
    __shared__ double s[kVecThreads / 32];
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) s[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = lane < kVecThreads / 32 ? s[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

// Called by every thread of every block after thread 0 stored partial[blockIdx.x].
// The last block to arrive reduces the partials in index order into *out.
__device__ void last_block_finalize(double* partial, unsigned* ticket, double* out, bool take_sqrt) {
    __shared__ bool is_last;
    __threadfence();
    if (threadIdx.x == 0) is_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double v = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) v += ((volatile double*)partial)[b];
    v = block_sum(v);
    if (threadIdx.x == 0) {
        *out = take_sqrt ? sqrt(v) : v;
        *ticket = 0u;
    }
}

__global__ void __launch_bounds__(kVecThreads) dot_kernel(const double* __restrict__ x, const double* __restrict__ y,
                                                          int64_t n, double* partial, unsigned* ticket, double* out,
                                                          int take_sqrt) {
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += x[i] * y[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
    last_block_finalize(partial, ticket, out, take_sqrt != 0);
}

__global__ void __launch_bounds__(kVecThreads) axpy_norm_kernel(const double* __restrict__ alpha,
                                                                const double* __restrict__ x, double* __restrict__ y,
                                                                int64_t n, double* partial, unsigned* ticket,
                                                                double* out) {
    const double a = *alpha;
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = y[i] - a * x[i];
        y[i] = v;
        acc += v * v;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
    last_block_finalize(partial, ticket, out, true);
}

// grid (nb, m): block (b, k) reduces its slice of <V_k, w> into partial[k * nb + b];
// the last block of row k to finish sums the row in index order into c[k]
// (tickets[k] counts the row's blocks and is reset).
__global__ void __launch_bounds__(kVecThreads) multidot_kernel(const double* __restrict__ V, int64_t ldv,
                                                               const double* __restrict__ w, int64_t n,
                                                               double* partial, unsigned* tickets,
                                                               double* __restrict__ c) {
    const int k = blockIdx.y;
    const double* v = V + (int64_t)k * ldv;
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += v[i] * w[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[(int64_t)k * gridDim.x + blockIdx.x] = acc;
    __shared__ bool is_last;
    __threadfence();
    if (threadIdx.x == 0) is_last = (atomicAdd(tickets + k, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double r = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
        r += ((volatile double*)partial)[(int64_t)k * gridDim.x + b];
    r = block_sum(r);
    if (threadIdx.x == 0) {
        c[k] = r;
        tickets[k] = 0u;
    }
}

// w = beta_w * w + sign * sum_k c[k] V_k; with `partial` non-null also the norm
// of the new w into *out (the reduction of dot_kernel(w, w): same slices, same
// order).
__global__ void __launch_bounds__(kVecThreads) combine_kernel(const double* __restrict__ V, int64_t ldv, int m,
                                                              const double* __restrict__ c, double sign,
                                                              double* __restrict__ w, double beta_w, int64_t n,
                                                              double* partial, unsigned* ticket, double* out) {
    __shared__ double cs[kMaxVec];
    for (int k = threadIdx.x; k < m; k += blockDim.x) cs[k] = sign * c[k];
    __syncthreads();
    double nrm = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double acc = beta_w == 0.0 ? 0.0 : beta_w * w[i];
        for (int k = 0; k < m; ++k) acc += cs[k] * V[(int64_t)k * ldv + i];
        w[i] = acc;
        nrm += acc * acc;
    }
    if (partial == nullptr) return;  // uniform
    nrm = block_sum(nrm);
    if (threadIdx.x == 0) partial[blockIdx.x] = nrm;
    last_block_finalize(partial, ticket, out, true);
}

__global__ void __launch_bounds__(kVecThreads) lanczos_shift_kernel(const double* __restrict__ beta,
                                                                    const double* __restrict__ v_cur,
                                                                    double* __restrict__ h,
                                                                    double* __restrict__ v_next, int64_t n) {
    const double b = *beta;
    const double inv = 1.0 / b;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        v_next[i] = h[i] * inv;
        h[i] = -b * v_cur[i];
    }
}

__global__ void __launch_bounds__(kVecThreads) scale_inv_kernel(double* __restrict__ x, const double* __restrict__ s,
                                                                int64_t n) {
    const double inv = 1.0 / *s;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] *= inv;
}

}  // namespace

int ReduceScratch::alloc(int blocks, int max_vectors) {
    max_blocks = blocks;
    DMRG_TRY(partial.alloc((size_t)blocks * (max_vectors > 0 ? max_vectors : 1) * sizeof(double)));
    if (!ticket.ptr) {
        DMRG_TRY(ticket.alloc((kRowTickets + kMaxVec) * sizeof(unsigned)));
        DMRG_TRY(ticket.zero());
    }
    return DMRG_OK;
}

int vec_dot(const double* x, const double* y, int64_t n, double* out, ReduceScratch& rs, int blocks,
            cudaStream_t st) {
    blocks = blocks < rs.max_blocks ? blocks : rs.max_blocks;
    dot_kernel<<<blocks, kVecThreads, 0, st>>>(x, y, n, rs.partial.as<double>(), rs.ticket.as<unsigned>(), out, 0);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_axpy_norm(const double* alpha, const double* x, double* y, int64_t n, double* out, ReduceScratch& rs,
                  int blocks, cudaStream_t st) {
    blocks = blocks < rs.max_blocks ? blocks : rs.max_blocks;
    axpy_norm_kernel<<<blocks, kVecThreads, 0, st>>>(alpha, x, y, n, rs.partial.as<double>(),
                                                     rs.ticket.as<unsigned>() + 1, out);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_multidot(const double* V, int64_t ldv, int m, const double* w, int64_t n, double* c, ReduceScratch& rs,
                 int blocks, cudaStream_t st) {
    if (m <= 0) return DMRG_OK;
    int nb = blocks / m;
    if (nb < 8) nb = 8;
    if (nb > rs.max_blocks) nb = rs.max_blocks;
    if ((size_t)nb * m * sizeof(double) > rs.partial.bytes)
        return set_error(DMRG_E_ARG, "multidot scratch too small (%d x %d)", nb, m);
    multidot_kernel<<<dim3(nb, m), kVecThreads, 0, st>>>(V, ldv, w, n, rs.partial.as<double>(),
                                                         rs.ticket.as<unsigned>() + kRowTickets, c);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_combine(const double* V, int64_t ldv, int m, const double* c, double sign, double* w, double beta_w,
                int64_t n, int blocks, cudaStream_t st) {
    if (m > kMaxVec) return set_error(DMRG_E_ARG, "combine of %d > %d vectors", m, kMaxVec);
    combine_kernel<<<blocks, kVecThreads, 0, st>>>(V, ldv, m, c, sign, w, beta_w, n, nullptr, nullptr, nullptr);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_lanczos_shift(const double* beta, const double* v_cur, double* h, double* v_next, int64_t n, int blocks,
                      cudaStream_t st) {
    lanczos_shift_kernel<<<blocks, kVecThreads, 0, st>>>(beta, v_cur, h, v_next, n);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_combine_normalize(const double* V, int64_t ldv, int m, const double* c, double sign, double* w, int64_t n,
                          double* out, ReduceScratch& rs, int blocks, cudaStream_t st) {
    if (m > kMaxVec) return set_error(DMRG_E_ARG, "combine of %d > %d vectors", m, kMaxVec);
    blocks = blocks < rs.max_blocks ? blocks : rs.max_blocks;
    combine_kernel<<<blocks, kVecThreads, 0, st>>>(V, ldv, m, c, sign, w, 1.0, n, rs.partial.as<double>(),
                                                   rs.ticket.as<unsigned>() + 2, out);
    scale_inv_kernel<<<blocks, kVecThreads, 0, st>>>(w, out, n);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_normalize(double* x, int64_t n, double* out, ReduceScratch& rs, int blocks, cudaStream_t st) {
    blocks = blocks < rs.max_blocks ? blocks : rs.max_blocks;
    dot_kernel<<<blocks, kVecThreads, 0, st>>>(x, x, n, rs.partial.as<double>(), rs.ticket.as<unsigned>() + 2, out,
                                               1);
    scale_inv_kernel<<<blocks, kVecThreads, 0, st>>>(x, out, n);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

}  // namespace dmrg
