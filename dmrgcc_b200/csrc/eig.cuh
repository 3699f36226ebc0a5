// Small dense FP64 eigen-solvers on the device (single CTA).
#pragma once

#include "common.cuh"

namespace dmrg {

// Lowest eigenvalue of the symmetric tridiagonal matrix (alpha[0..m), beta[0..m-1))
// by Sturm-count multisection, then the reference's Lanczos stopping test
// (real_tensor_lanczos.cc:110-112): state[0] = 1 when beta[m-1] < zero_tol,
// |E_m - E_{m-1}| < precision or m == niter; state[1] = m at that point.
// E[m-1] receives the eigenvalue.  Skips all work when state[0] is already set.
int launch_tridiag_lowest(const double* alpha, const double* beta, int m, double* E, int* state, double precision,
                          double zero_tol, int niter, cudaStream_t st);
// The same with m = *iter + 1 read on the device (graph-captured Lanczos loop).
int launch_tridiag_lowest_it(const double* alpha, const double* beta, const int* iter, double* E, int* state,
                             double precision, double zero_tol, int niter, cudaStream_t st);

// Cyclic parallel (round-robin) Jacobi eigensolver for a symmetric n x n matrix A
// (row-major, global memory, overwritten).  On return w[0..n) holds the
// eigenvalues in ascending order and Z (n x n, row-major) the eigenvectors as
// columns (Z[i*n + k] = component i of eigenvector k).  `ws` needs
// 2*n*n + 4*n doubles.  status[0] = DMRG_E_NUMERIC if 60 sweeps did not converge.
int launch_sym_jacobi(double* A, int n, double* w, double* Z, double* ws, int* status, cudaStream_t st);
// True when launch_sym_jacobi keeps an n x n problem in shared memory (its fast
// form); larger ones work in global memory, orders of magnitude slower.
bool sym_jacobi_in_shared(int n);

// Eigenvector y[0..m) of the tridiagonal (alpha, beta) of size *m_dev (read on
// the device: the Lanczos dimension is only known there) for its lowest
// eigenvalue E[m - 1], by inverse iteration; unit norm, largest component
// positive.  status[0] = DMRG_E_NUMERIC on m > 512 or a non-finite iterate.
int launch_tridiag_ground_vector(const double* alpha, const double* beta, const double* E, const int* m_dev,
                                 double* y, int* status, cudaStream_t st);

}  // namespace dmrg
