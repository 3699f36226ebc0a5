// Complex (interleaved re/im) vector kernels of the complex Lanczos solver
// (zvec.cu).  Vectors are n complex elements (2n doubles); scalars are complex
// (re, im) pairs unless stated.
#pragma once

#include "vec.cuh"

namespace dmrg {

struct ZReduce {
    DeviceBuffer partial;  // double2, >= blocks * max vectors
    DeviceBuffer ticket;
    DeviceBuffer scal;     // scratch scalars
    int max_blocks = 0;
    int alloc(int blocks, int max_vectors);
};

// out[0..1] = <x|y> = sum conj(x_i) y_i
int zvec_dot(const double* x, const double* y, int64_t n, double* out, ZReduce& rs, int blocks, cudaStream_t st);
// y -= alpha x (alpha complex, on the device);  *beta = sqrt(Re <y|y>) (real)
int zvec_axpy_norm(const double* alpha, const double* x, double* y, int64_t n, double* beta, ZReduce& rs, int blocks,
                   cudaStream_t st);
// c[k] = <V_k|w> (complex) for k < m   (V row-major m x n complex, leading dim ldv complex)
int zvec_multidot(const double* V, int64_t ldv, int m, const double* w, int64_t n, double* c, ZReduce& rs, int blocks,
                  cudaStream_t st);
// w -= sum_k c[k] V_k   (c complex, on the device)
int zvec_combine(const double* V, int64_t ldv, int m, const double* c, double* w, int64_t n, int blocks,
                 cudaStream_t st);

}  // namespace dmrg
