// FP64 vector kernels (see vec.cuh).  These are HBM-bound: each reads its
// operands once with coalesced grid-stride loops and reduces deterministically.
#include <algorithm>

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

// ---------------------------------------------------------------------------
// Device-indexed forms for the graph-captured Lanczos loop: the iteration i is
// read from state[kIterSlot] instead of being baked into launch arguments, so
// one captured iteration body serves every i.  Each computes exactly what its
// host-indexed twin above computes for that i (same slices, same reduction
// order, same effective grid), so a graph run is bit-identical to a launch-by-
// launch run.  Every kernel returns at once when state[0] (converged) is set.

__global__ void __launch_bounds__(kVecThreads) dot_it_kernel(const double* __restrict__ x,
                                                             const double* __restrict__ y, int64_t n,
                                                             double* partial, unsigned* ticket,
                                                             double* out_base, const int* state) {
    if (state[0]) return;
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc += x[i] * y[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
    last_block_finalize(partial, ticket, out_base + state[kIterSlot], false);
}

__global__ void __launch_bounds__(kVecThreads) axpy_norm_it_kernel(const double* __restrict__ alpha_base,
                                                                   const double* __restrict__ x,
                                                                   double* __restrict__ y, int64_t n,
                                                                   double* partial, unsigned* ticket,
                                                                   double* out_base, const int* state) {
    if (state[0]) return;
    const int it = state[kIterSlot];
    const double a = alpha_base[it];
    double acc = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = y[i] - a * x[i];
        y[i] = v;
        acc += v * v;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
    last_block_finalize(partial, ticket, out_base + it, true);
}

// v_next = V + (i+1) ldv = h / beta_i ; h = -beta_i x
__global__ void __launch_bounds__(kVecThreads) lanczos_shift_it_kernel(const double* __restrict__ beta_base,
                                                                       const double* __restrict__ x,
                                                                       double* __restrict__ h, double* V,
                                                                       int64_t ldv, int64_t n, int niter,
                                                                       const int* state) {
    if (state[0]) return;
    const int it = state[kIterSlot];
    if (it + 1 >= niter) return;
    double* __restrict__ v_next = V + (int64_t)(it + 1) * ldv;
    const double b = beta_base[it];
    const double inv = 1.0 / b;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        v_next[i] = h[i] * inv;
        h[i] = -b * x[i];
    }
}

// Number of slices of each vector in the multidot of m vectors:
// clamp(blocks / m, 8, max_blocks) (the host-indexed multidot's grid width).
__host__ __device__ __forceinline__ int multidot_slices(int blocks, int max_blocks, int m) {
    int nb = blocks / m;
    if (nb < 8) nb = 8;
    if (nb > max_blocks) nb = max_blocks;
    return nb;
}

// c[k] = <V_k, w> for k < m = i+1, w = V_{i+1}.  The host-indexed multidot runs
// an (nb, m) grid; here that grid is flattened into a 1-D grid sized for the
// largest nb * m of any iteration (multidot_it_grid): block j takes slice
// b = j % nb of vector k = j / nb, blocks with k >= m return.  Same slices,
// partials, tickets and reduction order as there.
__global__ void __launch_bounds__(kVecThreads) multidot_it_kernel(const double* __restrict__ V, int64_t ldv,
                                                                  int64_t n, int blocks, int max_blocks,
                                                                  double* partial, unsigned* tickets,
                                                                  double* __restrict__ c, int niter,
                                                                  const int* state) {
    if (state[0]) return;
    const int it = state[kIterSlot];
    if (it + 1 >= niter) return;
    const int m = it + 1;
    const int nb = multidot_slices(blocks, max_blocks, m);
    const int k = (int)blockIdx.x / nb, b = (int)blockIdx.x % nb;
    if (k >= m) return;
    const double* __restrict__ w = V + (int64_t)m * ldv;
    const double* __restrict__ v = V + (int64_t)k * ldv;
    double acc = 0.0;
    for (int64_t i = (int64_t)b * blockDim.x + threadIdx.x; i < n; i += (int64_t)nb * blockDim.x) acc += v[i] * w[i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) partial[(int64_t)k * nb + b] = acc;
    __shared__ bool is_last;
    __threadfence();
    if (threadIdx.x == 0) is_last = (atomicAdd(tickets + k, 1u) == (unsigned)nb - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double r = 0.0;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) r += ((volatile double*)partial)[(int64_t)k * nb + j];
    r = block_sum(r);
    if (threadIdx.x == 0) {
        c[k] = r;
        tickets[k] = 0u;
    }
}

// Grid of multidot_it_kernel: the largest nb * m over the iterations m < niter.
int multidot_it_grid(int blocks, int max_blocks, int niter) {
    int g = 1;
    for (int m = 1; m < niter; ++m) g = std::max(g, multidot_slices(blocks, max_blocks, m) * m);
    return g;
}

// w = V_{i+1} (+)= sign * sum_{k<=i} c[k] V_k; with `partial` also ||w|| into *out
__global__ void __launch_bounds__(kVecThreads) combine_it_kernel(const double* __restrict__ V, int64_t ldv,
                                                                 const double* __restrict__ c, double sign,
                                                                 int64_t n, double* partial, unsigned* ticket,
                                                                 double* out, int niter, const int* state) {
    if (state[0]) return;
    const int it = state[kIterSlot];
    if (it + 1 >= niter) return;
    const int m = it + 1;
    double* __restrict__ w = const_cast<double*>(V) + (int64_t)m * ldv;
    __shared__ double cs[kMaxVec];
    for (int k = threadIdx.x; k < m; k += blockDim.x) cs[k] = sign * c[k];
    __syncthreads();
    double nrm = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double acc = 1.0 * w[i];
        for (int k = 0; k < m; ++k) acc += cs[k] * V[(int64_t)k * ldv + i];
        w[i] = acc;
        nrm += acc * acc;
    }
    if (partial == nullptr) return;  // uniform
    nrm = block_sum(nrm);
    if (threadIdx.x == 0) partial[blockIdx.x] = nrm;
    last_block_finalize(partial, ticket, out, true);
}

// V_{i+1} /= *s, and the normalised vector also into x (the next matvec input)
__global__ void __launch_bounds__(kVecThreads) scale_inv_it_kernel(double* V, int64_t ldv,
                                                                   const double* __restrict__ s,
                                                                   double* __restrict__ x, int64_t n, int niter,
                                                                   const int* state) {
    if (state[0]) return;
    const int it = state[kIterSlot];
    if (it + 1 >= niter) return;
    double* __restrict__ w = V + (int64_t)(it + 1) * ldv;
    const double inv = 1.0 / *s;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = w[i] * inv;
        w[i] = v;
        x[i] = v;
    }
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
    DMRG_LAUNCH dot_kernel<<<blocks, kVecThreads, 0, st>>>(x, y, n, rs.partial.as<double>(), rs.ticket.as<unsigned>(), out, 0);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_axpy_norm(const double* alpha, const double* x, double* y, int64_t n, double* out, ReduceScratch& rs,
                  int blocks, cudaStream_t st) {
    blocks = blocks < rs.max_blocks ? blocks : rs.max_blocks;
    DMRG_LAUNCH axpy_norm_kernel<<<blocks, kVecThreads, 0, st>>>(alpha, x, y, n, rs.partial.as<double>(),
                                                     rs.ticket.as<unsigned>() + 1, out);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_multidot(const double* V, int64_t ldv, int m, const double* w, int64_t n, double* c, ReduceScratch& rs,
                 int blocks, cudaStream_t st) {
    if (m <= 0) return DMRG_OK;
    const int nb = multidot_slices(blocks, rs.max_blocks, m);
    if ((size_t)nb * m * sizeof(double) > rs.partial.bytes)
        return set_error(DMRG_E_ARG, "multidot scratch too small (%d x %d)", nb, m);
    DMRG_LAUNCH multidot_kernel<<<dim3(nb, m), kVecThreads, 0, st>>>(V, ldv, w, n, rs.partial.as<double>(),
                                                         rs.ticket.as<unsigned>() + kRowTickets, c);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_combine(const double* V, int64_t ldv, int m, const double* c, double sign, double* w, double beta_w,
                int64_t n, int blocks, cudaStream_t st) {
    if (m > kMaxVec) return set_error(DMRG_E_ARG, "combine of %d > %d vectors", m, kMaxVec);
    DMRG_LAUNCH combine_kernel<<<blocks, kVecThreads, 0, st>>>(V, ldv, m, c, sign, w, beta_w, n, nullptr, nullptr, nullptr);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_lanczos_shift(const double* beta, const double* v_cur, double* h, double* v_next, int64_t n, int blocks,
                      cudaStream_t st) {
    DMRG_LAUNCH lanczos_shift_kernel<<<blocks, kVecThreads, 0, st>>>(beta, v_cur, h, v_next, n);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_combine_normalize(const double* V, int64_t ldv, int m, const double* c, double sign, double* w, int64_t n,
                          double* out, ReduceScratch& rs, int blocks, cudaStream_t st) {
    if (m > kMaxVec) return set_error(DMRG_E_ARG, "combine of %d > %d vectors", m, kMaxVec);
    blocks = blocks < rs.max_blocks ? blocks : rs.max_blocks;
    DMRG_LAUNCH combine_kernel<<<blocks, kVecThreads, 0, st>>>(V, ldv, m, c, sign, w, 1.0, n, rs.partial.as<double>(),
                                                   rs.ticket.as<unsigned>() + 2, out);
    DMRG_LAUNCH scale_inv_kernel<<<blocks, kVecThreads, 0, st>>>(w, out, n);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_normalize(double* x, int64_t n, double* out, ReduceScratch& rs, int blocks, cudaStream_t st) {
    blocks = blocks < rs.max_blocks ? blocks : rs.max_blocks;
    DMRG_LAUNCH dot_kernel<<<blocks, kVecThreads, 0, st>>>(x, x, n, rs.partial.as<double>(), rs.ticket.as<unsigned>() + 2, out,
                                               1);
    DMRG_LAUNCH scale_inv_kernel<<<blocks, kVecThreads, 0, st>>>(x, out, n);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_dot_it(const double* x, const double* y, int64_t n, double* out_base, const int* state, ReduceScratch& rs,
               int blocks, cudaStream_t st) {
    blocks = blocks < rs.max_blocks ? blocks : rs.max_blocks;
    DMRG_LAUNCH dot_it_kernel<<<blocks, kVecThreads, 0, st>>>(x, y, n, rs.partial.as<double>(),
                                                              rs.ticket.as<unsigned>(), out_base, state);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_axpy_norm_it(const double* alpha_base, const double* x, double* y, int64_t n, double* out_base,
                     const int* state, ReduceScratch& rs, int blocks, cudaStream_t st) {
    blocks = blocks < rs.max_blocks ? blocks : rs.max_blocks;
    DMRG_LAUNCH axpy_norm_it_kernel<<<blocks, kVecThreads, 0, st>>>(alpha_base, x, y, n, rs.partial.as<double>(),
                                                                    rs.ticket.as<unsigned>() + 1, out_base, state);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int vec_lanczos_step_it(const double* beta_base, const double* x, double* h, double* V, int64_t n, int niter,
                        double* c, double* tmp, double* x_next, const int* state, ReduceScratch& rs, int blocks,
                        cudaStream_t st) {
    if (niter > kMaxVec) return set_error(DMRG_E_ARG, "Lanczos dimension %d > %d", niter, kMaxVec);
    if ((size_t)rs.max_blocks * niter * sizeof(double) > rs.partial.bytes)
        return set_error(DMRG_E_ARG, "multidot scratch too small (%d x %d)", rs.max_blocks, niter);
    const int cb = blocks < rs.max_blocks ? blocks : rs.max_blocks;
    unsigned* rows = rs.ticket.as<unsigned>() + kRowTickets;
    const int mg = multidot_it_grid(blocks, rs.max_blocks, niter);
    DMRG_LAUNCH lanczos_shift_it_kernel<<<blocks, kVecThreads, 0, st>>>(beta_base, x, h, V, n, n, niter, state);
    // classical Gram-Schmidt twice; the second pass also normalises
    DMRG_LAUNCH multidot_it_kernel<<<mg, kVecThreads, 0, st>>>(V, n, n, blocks, rs.max_blocks,
                                                                          rs.partial.as<double>(), rows, c, niter,
                                                                          state);
    DMRG_LAUNCH combine_it_kernel<<<blocks, kVecThreads, 0, st>>>(V, n, c, -1.0, n, nullptr, nullptr, nullptr, niter,
                                                                  state);
    DMRG_LAUNCH multidot_it_kernel<<<mg, kVecThreads, 0, st>>>(V, n, n, blocks, rs.max_blocks,
                                                                          rs.partial.as<double>(), rows, c, niter,
                                                                          state);
    DMRG_LAUNCH combine_it_kernel<<<cb, kVecThreads, 0, st>>>(V, n, c, -1.0, n, rs.partial.as<double>(),
                                                              rs.ticket.as<unsigned>() + 2, tmp, niter, state);
    DMRG_LAUNCH scale_inv_it_kernel<<<cb, kVecThreads, 0, st>>>(V, n, tmp, x_next, n, niter, state);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

}  // namespace dmrg
