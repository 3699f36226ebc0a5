// FP64 vector kernels for the Lanczos recurrence and reorthogonalisation.
// All reductions are deterministic: fixed per-block slices, partials reduced
// in index order by the last block to finish (atomic ticket).
#pragma once

#include "common.cuh"

namespace dmrg {

constexpr int kVecThreads = 256;

// Scratch shared by the reductions of one context/solver.
struct ReduceScratch {
    DeviceBuffer partial;  // doubles, >= kMaxBlocks * kMaxVec
    DeviceBuffer ticket;   // unsigned counters
    int max_blocks = 0;
    int alloc(int blocks, int max_vectors);
};

// out[0] = <x, y>
int vec_dot(const double* x, const double* y, int64_t n, double* out, ReduceScratch& rs, int blocks,
            cudaStream_t st);
// y -= (*alpha) * x ; out[0] = sqrt(||y||^2)
int vec_axpy_norm(const double* alpha, const double* x, double* y, int64_t n, double* out, ReduceScratch& rs,
                  int blocks, cudaStream_t st);
// c[k] = <V_k, w> for k < m   (V row-major m x n, leading dim ldv)
int vec_multidot(const double* V, int64_t ldv, int m, const double* w, int64_t n, double* c, ReduceScratch& rs,
                 int blocks, cudaStream_t st);
// w = beta_w * w + sign * sum_k c[k] V_k   (c on the device, m <= kMaxVec)
int vec_combine(const double* V, int64_t ldv, int m, const double* c, double sign, double* w, double beta_w,
                int64_t n, int blocks, cudaStream_t st);
// Lanczos step: v_next = h / beta ; h = -beta * v_cur   (beta on the device)
int vec_lanczos_shift(const double* beta, const double* v_cur, double* h, double* v_next, int64_t n, int blocks,
                      cudaStream_t st);
// w = w + sign * sum_k c[k] V_k, then w /= ||w|| (norm written to out[0]): the
// same arithmetic as vec_combine followed by vec_normalize, in two kernels
int vec_combine_normalize(const double* V, int64_t ldv, int m, const double* c, double sign, double* w, int64_t n,
                          double* out, ReduceScratch& rs, int blocks, cudaStream_t st);
// x /= ||x|| (two kernels: norm then scale); norm written to out[0]
int vec_normalize(double* x, int64_t n, double* out, ReduceScratch& rs, int blocks, cudaStream_t st);

constexpr int kMaxVec = 512;
constexpr int kRowTickets = 64;  // ticket slots before the per-row ones of vec_multidot

// ---- device-indexed Lanczos steps (for the graph-captured loop) -------------
// The iteration i is read from state[kIterSlot]; state[0] != 0 (converged)
// turns every call into a no-op.  The Krylov basis V is niter x n (ldv = n).
constexpr int kIterSlot = 4;
// out_base[i] = <x, y>
int vec_dot_it(const double* x, const double* y, int64_t n, double* out_base, const int* state, ReduceScratch& rs,
               int blocks, cudaStream_t st);
// y -= alpha_base[i] * x ; out_base[i] = ||y||
int vec_axpy_norm_it(const double* alpha_base, const double* x, double* y, int64_t n, double* out_base,
                     const int* state, ReduceScratch& rs, int blocks, cudaStream_t st);
// unless i + 1 == niter: V_{i+1} = h / beta_base[i], h = -beta_base[i] x; V_{i+1}
// orthogonalised against V_0..V_i by classical Gram-Schmidt twice (c: niter
// scratch doubles) and normalised (norm into *tmp); x_next = V_{i+1}.  The same
// arithmetic as vec_lanczos_shift + 2 x (vec_multidot, vec_combine[_normalize]).
int vec_lanczos_step_it(const double* beta_base, const double* x, double* h, double* V, int64_t n, int niter,
                        double* c, double* tmp, double* x_next, const int* state, ReduceScratch& rs, int blocks,
                        cudaStream_t st);

}  // namespace dmrg
