// Small dense FP64 eigen-solvers on the device (see eig.cuh).
//
// Tridiagonal lowest eigenvalue: Sturm sequence counts (number of negative
// pivots of the LDL^T factorisation of T - xI) evaluated at 128 points per
// round by one CTA (multisection), starting from the Gershgorin interval.
// Dense symmetric eigenproblem: two-sided cyclic Jacobi with the round-robin
// (Brent-Luk) ordering, n/2 disjoint rotations applied per round.
#include <cfloat>
#include <mutex>

#include "eig.cuh"

namespace dmrg {
namespace {

constexpr int kBisectThreads = 128;
constexpr int kJacobiThreads = 256;

__device__ int sturm_count(const double* alpha, const double* beta, int m, double x, double pivmin) {
    double d = alpha[0] - x;
    if (fabs(d) < pivmin) d = -pivmin;
    int cnt = d < 0.0;
    for (int k = 1; k < m; ++k) {
        const double b = beta[k - 1];
        d = (alpha[k] - x) - b * b / d;
        if (fabs(d) < pivmin) d = -pivmin;
        cnt += d < 0.0;
    }
    return cnt;
}

__global__ void __launch_bounds__(kBisectThreads) tridiag_lowest_kernel(const double* __restrict__ alpha,
                                                                         const double* __restrict__ beta, int m,
                                                                         double* __restrict__ E, int* state,
                                                                         double precision, double zero_tol,
                                                                         int niter, const int* m_iter) {
    __shared__ double lo, hi, pivmin;
    __shared__ int first;
    if (state[0]) return;  // already converged: later speculative steps are no-ops
    if (m_iter) m = *m_iter + 1;  // graph-captured loop: the dimension is the device's iteration + 1
    if (threadIdx.x == 0) {
        double l = DBL_MAX, h = -DBL_MAX, bmax = 0.0;
        for (int k = 0; k < m; ++k) {
            const double r = (k > 0 ? fabs(beta[k - 1]) : 0.0) + (k + 1 < m ? fabs(beta[k]) : 0.0);
            l = fmin(l, alpha[k] - r);
            h = fmax(h, alpha[k] + r);
            if (k + 1 < m) bmax = fmax(bmax, beta[k] * beta[k]);
        }
        const double span = fmax(fabs(l), fabs(h));
        lo = l - 2.0 * DBL_EPSILON * span - DBL_MIN;
        hi = h + 2.0 * DBL_EPSILON * span + DBL_MIN;
        pivmin = DBL_MIN * fmax(1.0, bmax);
    }
    __syncthreads();
    for (int round = 0; round < 64; ++round) {
        const double a = lo, b = hi;
        if (b - a <= 2.0 * DBL_EPSILON * fmax(fabs(a), fabs(b)) + DBL_MIN) break;
        if (threadIdx.x == 0) first = kBisectThreads;
        __syncthreads();
        const double x = a + (b - a) * (double)(threadIdx.x + 1) / (double)(kBisectThreads + 1);
        if (sturm_count(alpha, beta, m, x, pivmin) >= 1) atomicMin(&first, (int)threadIdx.x);
        __syncthreads();
        if (threadIdx.x == 0) {
            const int f = first;
            const double w = (b - a) / (double)(kBisectThreads + 1);
            lo = f == 0 ? a : a + w * (double)f;
            hi = f == kBisectThreads ? b : a + w * (double)(f + 1);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double lam = 0.5 * (lo + hi);
        E[m - 1] = lam;
        const double prev = m >= 2 ? E[m - 2] : 10000.0;  // old_energy starts at 10000 (real_tensor_lanczos.cc:76)
        if (beta[m - 1] < zero_tol || fabs(lam - prev) < precision || m == niter) {
            state[0] = 1;
            state[1] = m;
        }
    }
}

__device__ void round_robin_pair(int r, int i, int N, int& p, int& q) {
    // Circle method: player 0 fixed, players 1..N-1 rotate.
    if (i == 0) {
        p = 0;
        q = r % (N - 1) + 1;
    } else {
        p = (r + i) % (N - 1) + 1;
        q = (r - i + (N - 1)) % (N - 1) + 1;
    }
    if (p > q) {
        int t = p;
        p = q;
        q = t;
    }
}

__device__ double block_sum_j(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r += sh[k];
    __syncthreads();
    if (threadIdx.x == 0) sh[0] = r;
    __syncthreads();
    r = sh[0];
    __syncthreads();
    return r;
}

// Jacobi on A (n x n, global, row-major); Z accumulates the rotations (starts as I).
// cs: 2*ceil(n/2) doubles, pq: 2*ceil(n/2) ints (shared).
__device__ bool jacobi_core(double* A, int n, double* Z) {
    __shared__ double sh[kJacobiThreads / 32];
    extern __shared__ double dyn[];
    const int N = n + (n & 1);
    const int npair = N / 2;
    double* cs = dyn;                          // [npair][2]
    int* pq = reinterpret_cast<int*>(dyn + 2 * npair);  // [npair][2]
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) Z[idx] = (idx / n == idx % n) ? 1.0 : 0.0;
    __syncthreads();
    if (n <= 1) return true;
    bool converged = false;
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0.0, dia = 0.0;
        for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
            const int i = idx / n, j = idx % n;
            const double v = A[idx];
            if (i == j) dia += v * v;
            else off += v * v;
        }
        off = block_sum_j(off, sh);
        dia = block_sum_j(dia, sh);
        if (off <= 1e-28 * dia || off == 0.0) {  // off-diagonal mass below ~1e-14 of the diagonal
            converged = true;
            break;
        }
        for (int r = 0; r < N - 1; ++r) {
            for (int i = threadIdx.x; i < npair; i += blockDim.x) {
                int p, q;
                round_robin_pair(r, i, N, p, q);
                double c = 1.0, s = 0.0;
                if (q < n) {
                    const double apq = A[p * n + q];
                    if (apq != 0.0) {
                        const double tau = (A[q * n + q] - A[p * n + p]) / (2.0 * apq);
                        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                        c = 1.0 / sqrt(1.0 + t * t);
                        s = t * c;
                    }
                }
                cs[2 * i] = c;
                cs[2 * i + 1] = s;
                pq[2 * i] = p;
                pq[2 * i + 1] = q;
            }
            __syncthreads();
            // rows: A <- J^T A
            for (int idx = threadIdx.x; idx < npair * n; idx += blockDim.x) {
                const int i = idx / n, j = idx % n;
                const int p = pq[2 * i], q = pq[2 * i + 1];
                const double s = cs[2 * i + 1];
                if (q >= n || s == 0.0) continue;
                const double c = cs[2 * i];
                const double ap = A[p * n + j], aq = A[q * n + j];
                A[p * n + j] = c * ap - s * aq;
                A[q * n + j] = s * ap + c * aq;
            }
            __syncthreads();
            // columns: A <- A J, Z <- Z J
            for (int idx = threadIdx.x; idx < npair * n; idx += blockDim.x) {
                const int i = idx / n, row = idx % n;
                const int p = pq[2 * i], q = pq[2 * i + 1];
                const double s = cs[2 * i + 1];
                if (q >= n || s == 0.0) continue;
                const double c = cs[2 * i];
                const double ap = A[row * n + p], aq = A[row * n + q];
                A[row * n + p] = c * ap - s * aq;
                A[row * n + q] = s * ap + c * aq;
                const double zp = Z[row * n + p], zq = Z[row * n + q];
                Z[row * n + p] = c * zp - s * zq;
                Z[row * n + q] = s * zp + c * zq;
            }
            __syncthreads();
        }
    }
    return converged;
}

// Sign convention for an eigenvector (stride `stride`): its largest-magnitude
// component is positive; components within a relative 1e-6 of the largest
// count as equal and the first of them decides.  Sequential (n is small).
__device__ double eigvec_sign(const double* v, int n, int stride) {
    double mx = 0.0;
    for (int i = 0; i < n; ++i) mx = fmax(mx, fabs(v[(int64_t)i * stride]));
    if (mx == 0.0) return 1.0;
    for (int i = 0; i < n; ++i)
        if (fabs(v[(int64_t)i * stride]) >= mx * (1.0 - 1e-6)) return v[(int64_t)i * stride] < 0.0 ? -1.0 : 1.0;
    return 1.0;
}

// Dynamic shared memory of the solve: the rotation table (3 * npair doubles,
// jacobi_core's), then, when they fit, the working copies of A and Z, so that
// the thousands of barrier-separated passes of a solve stay on the SM.
constexpr size_t kJacobiSmemCap = 200 * 1024;
__host__ __device__ inline size_t jacobi_table_doubles(int n) { return (size_t)3 * ((n + (n & 1)) / 2); }
__host__ __device__ inline bool jacobi_in_smem(int n) {
    return (jacobi_table_doubles(n) + 2 * (size_t)n * n) * sizeof(double) <= kJacobiSmemCap;
}

__global__ void __launch_bounds__(kJacobiThreads) sym_jacobi_kernel(double* Ag, int n, double* w, double* Zout,
                                                                    double* ws, int* status) {
    extern __shared__ double dyn[];
    const bool local = jacobi_in_smem(n);
    double* A = local ? dyn + jacobi_table_doubles(n) : Ag;
    double* Z = local ? A + (size_t)n * n : ws;
    int* order = reinterpret_cast<int*>(ws + (size_t)n * n);
    if (local) {
        for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) A[idx] = Ag[idx];
        __syncthreads();
    }
    const bool ok = jacobi_core(A, n, Z);
    if (threadIdx.x == 0) {
        if (!ok) status[0] = DMRG_E_NUMERIC;
        for (int i = 0; i < n; ++i) order[i] = i;
        for (int i = 1; i < n; ++i) {  // stable insertion sort by eigenvalue, ascending
            const int key = order[i];
            const double kv = A[key * n + key];
            int j = i - 1;
            while (j >= 0 && A[order[j] * n + order[j]] > kv) {
                order[j + 1] = order[j];
                --j;
            }
            order[j + 1] = key;
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) w[k] = A[order[k] * n + order[k]];
    for (int idx = threadIdx.x; idx < n * n; idx += blockDim.x) {
        const int i = idx / n, k = idx % n;
        Zout[idx] = Z[i * n + order[k]];
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x)  // one column per thread
        if (eigvec_sign(Zout + k, n, n) < 0.0)
            for (int i = 0; i < n; ++i) Zout[i * n + k] = -Zout[i * n + k];
}

// Ground vector of the Lanczos tridiagonal T (alpha, beta; size *m_dev) by
// inverse iteration at its lowest eigenvalue lam = E[m - 1] (from the
// bisection, accurate to rounding): T - lam I is factored once by Gaussian
// elimination with partial pivoting (the tridiagonal scheme of LAPACK's
// dgttrf: pivoting rows k, k+1 fills a second superdiagonal), pivots below
// eps * ||T||_1 are raised to that size (the matrix is singular to rounding by
// construction), and three solves starting from the vector of ones give the
// eigenvector (normalised; the sign convention of eigvec_sign).  One thread:
// the recurrences are serial and m <= kMaxVec.
constexpr int kTriMax = 512;
__global__ void __launch_bounds__(32) tridiag_vector_kernel(const double* __restrict__ alpha,
                                                            const double* __restrict__ beta,
                                                            const double* __restrict__ E, const int* m_dev,
                                                            double* y, int* status) {
    __shared__ double d[kTriMax], du[kTriMax], du2[kTriMax], dl[kTriMax], x[kTriMax];
    __shared__ unsigned char swp[kTriMax];
    if (threadIdx.x != 0) return;
    const int n = *m_dev;
    if (n <= 0 || n > kTriMax) {
        status[0] = DMRG_E_NUMERIC;
        return;
    }
    if (n == 1) {
        y[0] = 1.0;
        return;
    }
    const double lam = E[n - 1];
    double tnorm = 0.0;  // ||T||_1
    for (int k = 0; k < n; ++k) {
        d[k] = alpha[k] - lam;
        tnorm = fmax(tnorm, fabs(alpha[k]) + (k > 0 ? fabs(beta[k - 1]) : 0.0) + (k + 1 < n ? fabs(beta[k]) : 0.0));
        if (k + 1 < n) dl[k] = du[k] = beta[k];
    }
    const double tiny = DBL_EPSILON * fmax(tnorm, DBL_MIN);
    // factor: rows k and k+1 are swapped when the subdiagonal entry is larger
    for (int k = 0; k + 1 < n; ++k) {
        if (fabs(d[k]) >= fabs(dl[k])) {
            swp[k] = 0;
            const double f = d[k] != 0.0 ? dl[k] / d[k] : 0.0;
            dl[k] = f;
            d[k + 1] -= f * du[k];
            du2[k] = 0.0;
        } else {
            swp[k] = 1;
            const double f = d[k] / dl[k];
            d[k] = dl[k];
            dl[k] = f;
            const double t = du[k];
            du[k] = d[k + 1];
            d[k + 1] = t - f * d[k + 1];
            if (k + 2 < n) {
                du2[k] = du[k + 1];
                du[k + 1] = -f * du[k + 1];
            } else {
                du2[k] = 0.0;
            }
        }
    }
    for (int k = 0; k < n; ++k)
        if (fabs(d[k]) < tiny) d[k] = d[k] < 0.0 ? -tiny : tiny;
    for (int k = 0; k < n; ++k) x[k] = 1.0;
    for (int it = 0; it < 3; ++it) {
        for (int k = 0; k + 1 < n; ++k) {  // L solve, with the row swaps
            if (swp[k]) {
                const double t = x[k];
                x[k] = x[k + 1];
                x[k + 1] = t - dl[k] * x[k];
            } else {
                x[k + 1] -= dl[k] * x[k];
            }
        }
        x[n - 1] /= d[n - 1];  // U solve
        x[n - 2] = (x[n - 2] - du[n - 2] * x[n - 1]) / d[n - 2];
        for (int k = n - 3; k >= 0; --k) x[k] = (x[k] - du[k] * x[k + 1] - du2[k] * x[k + 2]) / d[k];
        double mx = 0.0;
        for (int k = 0; k < n; ++k) mx = fmax(mx, fabs(x[k]));
        if (!(mx > 0.0) || !isfinite(mx)) {
            status[0] = DMRG_E_NUMERIC;
            return;
        }
        for (int k = 0; k < n; ++k) x[k] /= mx;  // keeps the next solve in range
    }
    double nrm = 0.0;
    for (int k = 0; k < n; ++k) nrm += x[k] * x[k];
    const double sc = eigvec_sign(x, n, 1) / sqrt(nrm);
    for (int k = 0; k < n; ++k) y[k] = sc * x[k];
}

}  // namespace

int launch_tridiag_lowest(const double* alpha, const double* beta, int m, double* E, int* state, double precision,
                          double zero_tol, int niter, cudaStream_t st) {
    DMRG_LAUNCH tridiag_lowest_kernel<<<1, kBisectThreads, 0, st>>>(alpha, beta, m, E, state, precision, zero_tol, niter,
                                                                    nullptr);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int launch_tridiag_lowest_it(const double* alpha, const double* beta, const int* iter, double* E, int* state,
                             double precision, double zero_tol, int niter, cudaStream_t st) {
    DMRG_LAUNCH tridiag_lowest_kernel<<<1, kBisectThreads, 0, st>>>(alpha, beta, 1, E, state, precision, zero_tol, niter,
                                                                    iter);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

static size_t jacobi_smem(int n) {
    return (jacobi_table_doubles(n) + (jacobi_in_smem(n) ? 2 * (size_t)n * n : 0)) * sizeof(double);
}

bool sym_jacobi_in_shared(int n) { return jacobi_in_smem(n); }

int launch_sym_jacobi(double* A, int n, double* w, double* Z, double* ws, int* status, cudaStream_t st) {
    if (n <= 0) return DMRG_OK;
    const size_t smem = jacobi_smem(n);
    if (smem > 48 * 1024) {
        // The kernel's shared-memory allowance is process-wide: raise it under a
        // lock and never lower it, so that runs side by side (one per host
        // thread, each with its own n) cannot undercut each other's launch.
        static std::mutex mu;
        static size_t allowed[64] = {};  // per device
        int dev = 0;
        DMRG_CUDA_TRY(cudaGetDevice(&dev));
        if (dev < 0 || dev >= 64) return set_error(DMRG_E_ARG, "device ordinal %d not supported", dev);
        std::lock_guard<std::mutex> lock(mu);
        if (smem > allowed[dev]) {
            DMRG_CUDA_TRY(cudaFuncSetAttribute(sym_jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            allowed[dev] = smem;
        }
    }
    DMRG_LAUNCH sym_jacobi_kernel<<<1, kJacobiThreads, smem, st>>>(A, n, w, Z, ws, status);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int launch_tridiag_ground_vector(const double* alpha, const double* beta, const double* E, const int* m_dev,
                                 double* y, int* status, cudaStream_t st) {
    DMRG_LAUNCH tridiag_vector_kernel<<<1, 32, 0, st>>>(alpha, beta, E, m_dev, y, status);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

}  // namespace dmrg
