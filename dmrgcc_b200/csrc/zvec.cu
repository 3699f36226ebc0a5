// Complex (interleaved re/im) vector kernels of the complex Lanczos solver:
// the conjugated inner products and complex-coefficient updates of
// ComplexTensorLanczos (src/dmrg/complexdmrg/complex_tensor_lanczos.cc:
// VectorMultiply :162-169, VectorSubtraction :171-176, GramSchmidtMethod
// :178-192).  Operations with real coefficients (scaling by 1/beta, the
// -beta shift, the ground-vector sum with the real tridiagonal eigenvector)
// run through the real kernels on the 2n doubles.  Reductions are
// deterministic as in vec.cu: per-block partials summed in block order by the
// last block to finish.
#include "zvec.cuh"

namespace dmrg {
namespace {

constexpr int kT = kVecThreads;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Sums two values over the block; results valid in thread 0.
__device__ void block_sum2(double& a, double& b) {
    __shared__ double s[2][kT / 32];
    a = warp_sum(a);
    b = warp_sum(b);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        s[0][w] = a;
        s[1][w] = b;
    }
    __syncthreads();
    if (w == 0) {
        a = lane < kT / 32 ? s[0][lane] : 0.0;
        b = lane < kT / 32 ? s[1][lane] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
    }
    __syncthreads();
}

// The last block of the grid sums the (re, im) partials in block order into out.
__device__ void finalize2(double2* partial, unsigned* ticket, double2* out, int nb) {
    __shared__ bool is_last;
    __threadfence();
    if (threadIdx.x == 0) is_last = (atomicAdd(ticket, 1u) == (unsigned)nb - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double a = 0.0, b = 0.0;
    const volatile double* pv = reinterpret_cast<volatile double*>(partial);
    for (int k = threadIdx.x; k < nb; k += blockDim.x) {
        a += pv[2 * k];
        b += pv[2 * k + 1];
    }
    block_sum2(a, b);
    if (threadIdx.x == 0) {
        *out = make_double2(a, b);
        *ticket = 0u;
    }
}

// out = sum conj(x_i) y_i
__global__ void __launch_bounds__(kT) zdot_kernel(const double2* __restrict__ x, const double2* __restrict__ y,
                                                  int64_t n, double2* partial, unsigned* ticket, double2* out) {
    double re = 0.0, im = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 a = x[i], b = y[i];
        re += a.x * b.x + a.y * b.y;
        im += a.x * b.y - a.y * b.x;
    }
    block_sum2(re, im);
    if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(re, im);
    finalize2(partial, ticket, out, gridDim.x);
}

// y -= alpha x (complex alpha);  *sum = (<y|y>, 0)
__global__ void __launch_bounds__(kT) zaxpy_norm_kernel(const double2* __restrict__ alpha, const double2* __restrict__ x,
                                                        double2* __restrict__ y, int64_t n, double2* partial,
                                                        unsigned* ticket, double2* sum) {
    const double2 a = *alpha;
    double acc = 0.0, zero = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 u = x[i];
        double2 v = y[i];
        v.x -= a.x * u.x - a.y * u.y;
        v.y -= a.x * u.y + a.y * u.x;
        y[i] = v;
        acc += v.x * v.x + v.y * v.y;
    }
    block_sum2(acc, zero);
    if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(acc, 0.0);
    finalize2(partial, ticket, sum, gridDim.x);
}

// *out = sqrt(Re *s): beta = <h|h>^(1/2) as the reference takes it (:88)
__global__ void sqrt_re_kernel(const double2* __restrict__ s, double* __restrict__ out) { *out = sqrt(s->x); }

// c[k] = sum conj(V_k,i) w_i, k < m   (grid (nb, m), one row per blockIdx.y)
__global__ void __launch_bounds__(kT) zmultidot_kernel(const double2* __restrict__ V, int64_t ldv,
                                                       const double2* __restrict__ w, int64_t n, double2* partial,
                                                       unsigned* tickets, double2* __restrict__ c) {
    const int k = blockIdx.y;
    const double2* v = V + (int64_t)k * ldv;
    double re = 0.0, im = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 a = v[i], b = w[i];
        re += a.x * b.x + a.y * b.y;
        im += a.x * b.y - a.y * b.x;
    }
    block_sum2(re, im);
    if (threadIdx.x == 0) partial[(int64_t)k * gridDim.x + blockIdx.x] = make_double2(re, im);
    finalize2(partial + (int64_t)k * gridDim.x, tickets + k, c + k, gridDim.x);
}

// w -= sum_k c[k] V_k (complex c)
__global__ void __launch_bounds__(kT) zcombine_kernel(const double2* __restrict__ V, int64_t ldv, int m,
                                                      const double2* __restrict__ c, double2* __restrict__ w,
                                                      int64_t n) {
    __shared__ double2 cs[kMaxVec];
    for (int k = threadIdx.x; k < m; k += blockDim.x) cs[k] = c[k];
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double2 acc = w[i];
        for (int k = 0; k < m; ++k) {
            const double2 a = V[(int64_t)k * ldv + i], b = cs[k];
            acc.x -= b.x * a.x - b.y * a.y;
            acc.y -= b.x * a.y + b.y * a.x;
        }
        w[i] = acc;
    }
}

}  // namespace

int ZReduce::alloc(int blocks, int max_vectors) {
    max_blocks = blocks;
    DMRG_TRY(partial.alloc((size_t)blocks * (max_vectors > 0 ? max_vectors : 1) * sizeof(double2)));
    DMRG_TRY(scal.alloc(4 * sizeof(double2)));
    if (!ticket.ptr) {
        DMRG_TRY(ticket.alloc((4 + kMaxVec) * sizeof(unsigned)));
        DMRG_TRY(ticket.zero());
    }
    return DMRG_OK;
}

int zvec_dot(const double* x, const double* y, int64_t n, double* out, ZReduce& rs, int blocks, cudaStream_t st) {
    blocks = blocks < rs.max_blocks ? blocks : rs.max_blocks;
    DMRG_LAUNCH zdot_kernel<<<blocks, kT, 0, st>>>(reinterpret_cast<const double2*>(x),
                                                   reinterpret_cast<const double2*>(y), n, rs.partial.as<double2>(),
                                                   rs.ticket.as<unsigned>(), reinterpret_cast<double2*>(out));
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int zvec_axpy_norm(const double* alpha, const double* x, double* y, int64_t n, double* beta, ZReduce& rs, int blocks,
                   cudaStream_t st) {
    blocks = blocks < rs.max_blocks ? blocks : rs.max_blocks;
    double2* sum = rs.scal.as<double2>();
    DMRG_LAUNCH zaxpy_norm_kernel<<<blocks, kT, 0, st>>>(
        reinterpret_cast<const double2*>(alpha), reinterpret_cast<const double2*>(x), reinterpret_cast<double2*>(y), n,
        rs.partial.as<double2>(), rs.ticket.as<unsigned>() + 1, sum);
    DMRG_LAUNCH sqrt_re_kernel<<<1, 1, 0, st>>>(sum, beta);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int zvec_multidot(const double* V, int64_t ldv, int m, const double* w, int64_t n, double* c, ZReduce& rs, int blocks,
                  cudaStream_t st) {
    if (m <= 0) return DMRG_OK;
    int nb = blocks / m;
    if (nb < 8) nb = 8;
    if (nb > rs.max_blocks) nb = rs.max_blocks;
    if ((size_t)nb * m * sizeof(double2) > rs.partial.bytes)
        return set_error(DMRG_E_ARG, "complex multidot scratch too small (%d x %d)", nb, m);
    DMRG_LAUNCH zmultidot_kernel<<<dim3(nb, m), kT, 0, st>>>(
        reinterpret_cast<const double2*>(V), ldv, reinterpret_cast<const double2*>(w), n, rs.partial.as<double2>(),
        rs.ticket.as<unsigned>() + 4, reinterpret_cast<double2*>(c));
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int zvec_combine(const double* V, int64_t ldv, int m, const double* c, double* w, int64_t n, int blocks,
                 cudaStream_t st) {
    if (m > kMaxVec) return set_error(DMRG_E_ARG, "complex combine of %d > %d vectors", m, kMaxVec);
    DMRG_LAUNCH zcombine_kernel<<<blocks, kT, 0, st>>>(reinterpret_cast<const double2*>(V), ldv, m,
                                                       reinterpret_cast<const double2*>(c),
                                                       reinterpret_cast<double2*>(w), n);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

}  // namespace dmrg
