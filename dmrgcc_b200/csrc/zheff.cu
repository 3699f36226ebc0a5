// The complex path: complex128 H_eff * psi and its Lanczos ground state.
//
// ComplexTensorContraction::MultiplyEffectHamilton (src/dmrg/complexdmrg/
// complex_tensor_contraction.cc:1244-1312) is the real walk of heff.cu with
// complex blocks and a complex MPO: stage A T = K R, stage B out += w L T, on
// the complex grouped GEMM (zgemm.cu).  ComplexTensorLanczos::LanczosMethod
// (complex_tensor_lanczos.cc:14-160): alpha_i = <v_i|h> with the conjugated
// product, h -= alpha_i v_i with the complex alpha, beta_i = sqrt(Re <h|h>), the
// tridiagonal problem on Re alpha and beta (zheevd reads only the real diagonal
// of a Hermitian matrix), Gram-Schmidt with complex coefficients; the ground
// vector is the real tridiagonal eigenvector's combination.  psi_dim < 100:
// the dense branch (ComputeEffectHamilton + zheevd) on the real symmetric
// 2n x 2n form [[Re H, -Im H], [Im H, Re H]] of the Hermitian H, whose lowest
// eigenvector (x, y) gives the complex ground state x + i y.
#include <algorithm>
#include <cmath>

#include "blocksparse.h"
#include "eig.cuh"
#include "zgemm.cuh"
#include "zvec.cuh"

using namespace dmrg;

struct dmrg_zheff_s {
    dmrg_ctx_t ctx = nullptr;
    SiteDesc site;              // structure; site.W holds the real parts
    std::vector<double> Wc;     // complex MPO [lb][rb][d][d] (re, im)
    EnvDesc L, R;
    ZGemmSchedule sa, sb;
    DeviceBuffer T;
    int64_t t_size = 0;         // complex elements
    const double* L_dev = nullptr;
    const double* R_dev = nullptr;
    double flops_alg = 0;
    // Lanczos work
    int niter = 0;
    DeviceBuffer V, h, scal, state, y, dense, jac;
    ZReduce zr;
    ReduceScratch rs;
};

namespace {

inline double wre(const std::vector<double>& Wc, const SiteDesc& s, int o1, int o2, int p1, int p2) {
    return Wc[2 * ((((size_t)o1 * s.rb + o2) * s.d + p1) * s.d + p2)];
}
inline double wim(const std::vector<double>& Wc, const SiteDesc& s, int o1, int o2, int p1, int p2) {
    return Wc[2 * ((((size_t)o1 * s.rb + o2) * s.d + p1) * s.d + p2) + 1];
}

int build_zheff(dmrg_zheff_s& h) {
    const SiteDesc& s = h.site;
    const BlockListDesc& ket = s.ket;
    auto same_right = ket.by_sector(1, s.nr);
    for (int o = 0; o < s.lb; ++o)
        for (int q = 0; q < h.L.o[o].count(); ++q)
            if (h.L.o[o].left[q] < 0 || h.L.o[o].left[q] >= s.nl || h.L.o[o].right[q] < 0 ||
                h.L.o[o].right[q] >= s.nl)
                return set_error(DMRG_E_ARG, "L[%d] block %d has sectors outside %d", o, q, s.nl);
    for (int o = 0; o < s.rb; ++o)
        for (int q = 0; q < h.R.o[o].count(); ++q)
            if (h.R.o[o].left[q] < 0 || h.R.o[o].left[q] >= s.nr || h.R.o[o].right[q] < 0 ||
                h.R.o[o].right[q] >= s.nr)
                return set_error(DMRG_E_ARG, "R[%d] block %d has sectors outside %d", o, q, s.nr);
    // ComplexTensorOperator::RightCheckZero (complex_tensor_operator.cc:379-393): |w| > 1e-15
    auto right_nonzero = [&](int o2, int p2) {
        for (int o1 = 0; o1 < s.lb; ++o1)
            for (int p1 = 0; p1 < s.d; ++p1)
                if (std::hypot(wre(h.Wc, s, o1, o2, p1, p2), wim(h.Wc, s, o1, o2, p1, p2)) > 1e-15) return true;
        return false;
    };
    struct TermB {
        int out_pos;
        int64_t l_off;
        int lda, t_index, k;
        double wr, wi;
    };
    struct TaskA {
        int pos;
        int64_t r_off;
        int b_l, b_j, a_k;
        int64_t t_off;
    };
    std::vector<TermB> termsB;
    std::vector<TaskA> tasks;
    h.t_size = 0;
    double fl = 0;
    for (int o2 = 0; o2 < s.rb; ++o2) {
        const BlockListDesc& Ro = h.R.o[o2];
        for (int i = 0; i < Ro.count(); ++i) {
            const int ldx = Ro.left[i], jdx = Ro.right[i], rr = Ro.rows[i], rc = Ro.cols[i];
            if (rr == 0) continue;
            for (int pos : same_right[ldx]) {
                const int kdx = ket.left[pos];
                const int p2 = s.pb(pos);
                if (!right_nonzero(o2, p2)) continue;
                const int a_k = ket.rows[pos], b_l = ket.cols[pos];
                if (b_l != rr)
                    return set_error(DMRG_E_ARG, "ket block %d is %dx%d but R[%d] block %d is %dx%d", pos, a_k, b_l, o2,
                                     i, rr, rc);
                fl += 8.0 * a_k * b_l * rc;
                if (a_k == 0 || b_l == 0 || rc == 0) continue;
                const int t_index = (int)tasks.size();
                bool used = false;
                for (int pos2 : same_right[jdx]) {
                    const int idx = ket.left[pos2];
                    const int p1 = s.pb(pos2);
                    for (int o1 = 0; o1 < s.lb; ++o1) {
                        const double wr = wre(h.Wc, s, o1, o2, p1, p2), wi = wim(h.Wc, s, o1, o2, p1, p2);
                        if (wr == 0.0 && wi == 0.0) continue;
                        const int q = h.L.o[o1].find(idx, kdx);
                        if (q == -1) continue;
                        const int lr = h.L.o[o1].rows[q], lc = h.L.o[o1].cols[q];
                        if (lc != a_k || lr != ket.rows[pos2] || rc != ket.cols[pos2])
                            return set_error(DMRG_E_ARG, "shape mismatch in the complex H_eff at L[%d] block %d", o1, q);
                        if (lr == 0) continue;
                        termsB.push_back(TermB{pos2, h.L.base[o1] + h.L.o[o1].off[q], lc, t_index, a_k, wr, wi});
                        fl += 8.0 * lr * lc * rc;
                        used = true;
                    }
                }
                if (used) {
                    tasks.push_back(TaskA{pos, h.R.base[o2] + Ro.off[i], b_l, rc, a_k, h.t_size});
                    h.t_size += (int64_t)a_k * rc;
                }
            }
        }
    }
    h.sa.reset();
    for (const TaskA& t : tasks) {
        h.sa.add_group(t.t_off, t.b_j, t.a_k, t.b_j);
        h.sa.add_term(ket.off[t.pos], t.b_l, t.r_off, t.b_j, t.b_l, 1.0, 0.0);
    }
    h.sb.reset();
    std::vector<std::vector<int>> per_out(ket.count());
    for (int i = 0; i < (int)termsB.size(); ++i) per_out[termsB[i].out_pos].push_back(i);
    for (int pos2 = 0; pos2 < ket.count(); ++pos2) {
        if (per_out[pos2].empty()) continue;
        h.sb.add_group(ket.off[pos2], ket.cols[pos2], ket.rows[pos2], ket.cols[pos2]);
        for (int i : per_out[pos2]) {
            const TermB& t = termsB[i];
            const TaskA& ta = tasks[t.t_index];
            h.sb.add_term(t.l_off, t.lda, ta.t_off, ta.b_j, t.k, t.wr, t.wi);
        }
    }
    h.flops_alg = fl;
    DMRG_TRY(h.sa.check_bounds(ket.size, h.R.size, h.t_size));
    DMRG_TRY(h.sb.check_bounds(h.L.size, h.t_size, ket.size));
    DMRG_TRY(h.sa.finalize(h.ctx->stream));
    DMRG_TRY(h.sb.finalize(h.ctx->stream));
    DMRG_TRY(h.T.alloc((size_t)std::max<int64_t>(h.t_size, 1) * 2 * sizeof(double)));
    return DMRG_OK;
}

int zapply(dmrg_zheff_s& h, const double* psi, double* out, bool accumulate) {
    if ((!h.L_dev && h.L.size) || (!h.R_dev && h.R.size))
        return set_error(DMRG_E_STATE, "dmrg_zheff_set_env was not called");
    cudaStream_t st = h.ctx->stream;
    if (!accumulate && h.site.ket.size)
        DMRG_CUDA_TRY(cudaMemsetAsync(out, 0, (size_t)h.site.ket.size * 2 * sizeof(double), st));
    DMRG_TRY(launch_zgemm(h.sa, psi, h.R_dev, h.T.as<double>(), false, st));
    DMRG_TRY(launch_zgemm(h.sb, h.L_dev, h.T.as<double>(), out, true, st));
    return DMRG_OK;
}

__global__ void zunit_kernel(double* x, int64_t n, int64_t c) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < 2 * n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = i == 2 * c ? 1.0 : 0.0;
}

// cols[c*n + r] = (H e_c)[r] (complex) -> the real symmetric 2n x 2n form of H,
// H[r][c] from the upper triangle (r <= c) and conj(H[c][r]) below it.
__global__ void realify_kernel(const double2* __restrict__ cols, double* __restrict__ A, int n) {
    const int N = 2 * n;
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
        const int r = idx / n, c = idx % n;
        double2 v = r <= c ? cols[(int64_t)c * n + r] : cols[(int64_t)r * n + c];
        if (r > c) v.y = -v.y;
        A[(int64_t)r * N + c] = v.x;              // Re H
        A[(int64_t)r * N + n + c] = -v.y;         // -Im H
        A[(int64_t)(n + r) * N + c] = v.y;        // Im H
        A[(int64_t)(n + r) * N + n + c] = v.x;    // Re H
    }
}

// psi (complex) = z[0:n] + i z[n:2n] from column 0 of Z (2n x 2n, row-major)
__global__ void unrealify_kernel(const double* __restrict__ Z, int n, double* __restrict__ psi) {
    const int N = 2 * n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        psi[2 * i] = Z[(int64_t)i * N];
        psi[2 * i + 1] = Z[(int64_t)(n + i) * N];
    }
}

// alpha_re[i] = Re alpha_c[i]
__global__ void real_part_kernel(const double* __restrict__ zc, double* __restrict__ re) { *re = zc[0]; }

int ensure_zwork(dmrg_zheff_s& h, int niter) {
    const int64_t n = h.site.ket.size;
    if (h.niter < niter) {
        DMRG_TRY(h.V.alloc((size_t)std::max(niter, 1) * std::max<int64_t>(n, 1) * 2 * sizeof(double)));
        DMRG_TRY(h.h.alloc((size_t)std::max<int64_t>(n, 1) * 2 * sizeof(double)));
        DMRG_TRY(h.scal.alloc((size_t)(8 * std::max(niter, 1) + 16) * sizeof(double)));
        DMRG_TRY(h.y.alloc((size_t)std::max(niter, 1) * sizeof(double)));
        h.niter = niter;
    }
    DMRG_TRY(h.state.alloc(16 * sizeof(int)));
    DMRG_TRY(h.zr.alloc(std::max(2 * h.ctx->num_sms, 64), std::max(niter, 1)));
    DMRG_TRY(h.rs.alloc(std::max(2 * h.ctx->num_sms, 64), 1));
    return DMRG_OK;
}

int zexact(dmrg_zheff_s& h, double* psi, double* energy) {
    const int n = (int)h.site.ket.size;
    const int N = 2 * n;
    cudaStream_t st = h.ctx->stream;
    DMRG_TRY(h.dense.alloc((size_t)(2 * n * n + 2 * N * N + 4 * N + 8) * sizeof(double)));
    const int m = std::max(N, 128);
    DMRG_TRY(h.jac.alloc((size_t)(2 * m * m + 4 * m) * sizeof(double)));
    double* cols = h.dense.as<double>();
    double* A = cols + (size_t)2 * n * n;
    double* Z = A + (size_t)N * N;
    double* ev = Z + (size_t)N * N;
    double* e = h.h.as<double>();
    for (int c = 0; c < n; ++c) {
        DMRG_LAUNCH zunit_kernel<<<1, 128, 0, st>>>(e, n, c);
        DMRG_TRY(zapply(h, e, cols + (size_t)2 * c * n, false));
    }
    DMRG_LAUNCH realify_kernel<<<std::max(1, (n * n + 255) / 256), 256, 0, st>>>(reinterpret_cast<double2*>(cols), A, n);
    int* state = h.state.as<int>();
    DMRG_CUDA_TRY(cudaMemsetAsync(state, 0, 16 * sizeof(int), st));
    DMRG_TRY(launch_sym_jacobi(A, N, ev, Z, h.jac.as<double>(), state + 2, st));
    DMRG_LAUNCH unrealify_kernel<<<1, 128, 0, st>>>(Z, n, psi);
    double e0 = 0.0;
    int status[4] = {0, 0, 0, 0};
    DMRG_CUDA_TRY(cudaMemcpyAsync(&e0, ev, sizeof(double), cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaMemcpyAsync(status, state, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaStreamSynchronize(st));
    if (status[2] != 0) return set_error(DMRG_E_NUMERIC, "Jacobi eigensolver did not converge (2n=%d)", N);
    *energy = e0;
    return DMRG_OK;
}

int zkrylov(dmrg_zheff_s& h, double* psi, int niter, double precision, double zero_tol, double* energy, int* iters) {
    const int64_t n = h.site.ket.size;  // complex elements
    cudaStream_t st = h.ctx->stream;
    const int blocks = (int)std::min<int64_t>((n + kVecThreads - 1) / kVecThreads, 2 * h.ctx->num_sms);
    double* V = h.V.as<double>();
    double* hv = h.h.as<double>();
    double* alpha_c = h.scal.as<double>();   // 2 niter
    double* alpha = alpha_c + 2 * niter;     // niter
    double* beta = alpha + niter;
    double* E = beta + niter;
    double* c = E + niter;                   // 2 niter
    double* tmp = c + 2 * niter;
    int* state = h.state.as<int>();
    const int64_t ldv = 2 * n;  // doubles per vector
    DMRG_CUDA_TRY(cudaMemcpyAsync(V, psi, n * 2 * sizeof(double), cudaMemcpyDeviceToDevice, st));
    DMRG_CUDA_TRY(cudaMemsetAsync(hv, 0, n * 2 * sizeof(double), st));
    DMRG_CUDA_TRY(cudaMemsetAsync(state, 0, 16 * sizeof(int), st));
    int host_state[4] = {0, 0, 0, 0};
    const int chunk = (int)std::min<int64_t>(8, std::max<int64_t>(2, 1000000 / (n + 50000)));
    int dim = 0;
    for (int i = 0; i < niter; ++i) {
        double* vi = V + (int64_t)i * ldv;
        DMRG_TRY(zapply(h, vi, hv, true));
        DMRG_TRY(zvec_dot(vi, hv, n, alpha_c + 2 * i, h.zr, blocks, st));
        DMRG_TRY(zvec_axpy_norm(alpha_c + 2 * i, vi, hv, n, beta + i, h.zr, blocks, st));
        DMRG_LAUNCH real_part_kernel<<<1, 1, 0, st>>>(alpha_c + 2 * i, alpha + i);
        DMRG_TRY(launch_tridiag_lowest(alpha, beta, i + 1, E, state, precision, zero_tol, niter, st));
        if ((i + 1) % chunk == 0 || i + 1 == niter) {
            DMRG_CUDA_TRY(cudaMemcpyAsync(host_state, state, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
            DMRG_CUDA_TRY(cudaStreamSynchronize(st));
            if (host_state[0]) {
                dim = host_state[1];
                break;
            }
        }
        if (i + 1 == niter) break;
        double* vn = V + (int64_t)(i + 1) * ldv;
        // v_{i+1} = h / beta_i ; h = -beta_i v_i  (real coefficients: the real kernel on 2n doubles)
        DMRG_TRY(vec_lanczos_shift(beta + i, vi, hv, vn, 2 * n, blocks, st));
        // Gram-Schmidt with complex coefficients, twice, then normalise
        for (int pass = 0; pass < 2; ++pass) {
            DMRG_TRY(zvec_multidot(V, n, i + 1, vn, n, c, h.zr, blocks, st));
            DMRG_TRY(zvec_combine(V, n, i + 1, c, vn, n, blocks, st));
        }
        DMRG_TRY(vec_normalize(vn, 2 * n, tmp, h.rs, blocks, st));
    }
    if (dim <= 0) return set_error(DMRG_E_NUMERIC, "complex Lanczos ended without a converged dimension");
    DMRG_TRY(launch_tridiag_ground_vector(alpha, beta, E, state + 1, h.y.as<double>(), state + 2, st));
    DMRG_TRY(vec_combine(V, ldv, dim, h.y.as<double>(), 1.0, psi, 0.0, 2 * n, blocks, st));
    double e = 0.0;
    DMRG_CUDA_TRY(cudaMemcpyAsync(&e, E + dim - 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaMemcpyAsync(host_state, state, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaStreamSynchronize(st));
    if (host_state[2] != 0) return set_error(DMRG_E_NUMERIC, "tridiagonal ground vector failed (m=%d)", dim);
    *energy = e;
    if (iters) *iters = dim;
    return DMRG_OK;
}

}  // namespace

extern "C" {

int dmrg_zheff_create(dmrg_ctx_t ctx, int nl, int nr, const int* phys, const dmrg_blocks_t* ket, int d, int lb,
                      int rb, const double* W, const dmrg_blocks_t* L, const dmrg_blocks_t* R, dmrg_zheff_t* out) {
    if (!ctx || !out || !L || !R || !W || lb <= 0 || rb <= 0 || d <= 0) return set_error(DMRG_E_ARG, "null argument");
    *out = nullptr;
    DMRG_CUDA_TRY(cudaSetDevice(ctx->device));
    const size_t nw = (size_t)lb * rb * d * d;
    std::vector<double> wr(nw);
    for (size_t i = 0; i < nw; ++i) wr[i] = W[2 * i];
    auto* h = new dmrg_zheff_s();
    h->ctx = ctx;
    h->Wc.assign(W, W + 2 * nw);
    int rc = build_site_desc(h->site, nl, nr, phys, ket, d, lb, rb, wr.data());
    if (rc == DMRG_OK && !h->L.assign(L, lb)) rc = set_error(DMRG_E_ARG, "invalid L block lists");
    if (rc == DMRG_OK && !h->R.assign(R, rb)) rc = set_error(DMRG_E_ARG, "invalid R block lists");
    if (rc == DMRG_OK) rc = build_zheff(*h);
    if (rc != DMRG_OK) {
        delete h;
        return rc;
    }
    *out = h;
    return DMRG_OK;
}

int dmrg_zheff_destroy(dmrg_zheff_t h) {
    delete h;
    return DMRG_OK;
}

int dmrg_zheff_sizes(dmrg_zheff_t h, int64_t* psi_dim, int64_t* lsize, int64_t* rsize, double* flops) {
    if (!h) return set_error(DMRG_E_ARG, "null operator");
    if (psi_dim) *psi_dim = h->site.ket.size;
    if (lsize) *lsize = h->L.size;
    if (rsize) *rsize = h->R.size;
    if (flops) *flops = h->flops_alg;
    return DMRG_OK;
}

int dmrg_zheff_set_env(dmrg_zheff_t h, const double* L_dev, const double* R_dev) {
    if (!h) return set_error(DMRG_E_ARG, "null operator");
    if ((!L_dev && h->L.size) || (!R_dev && h->R.size)) return set_error(DMRG_E_ARG, "null environment pointer");
    h->L_dev = L_dev;
    h->R_dev = R_dev;
    return DMRG_OK;
}

int dmrg_zheff_apply(dmrg_zheff_t h, const double* psi, double* out, int accumulate) {
    if (!h) return set_error(DMRG_E_ARG, "null operator");
    return zapply(*h, psi, out, accumulate != 0);
}

int dmrg_zlanczos(dmrg_zheff_t h, double* psi, int niter, double precision, double zero_tol, double* energy,
                  int* iters) {
    if (!h || !psi || !energy || niter <= 0) return set_error(DMRG_E_ARG, "invalid Lanczos arguments");
    if (niter > kMaxVec) return set_error(DMRG_E_ARG, "niter %d above %d", niter, kMaxVec);
    DMRG_TRY(ensure_zwork(*h, niter));
    // The dense branch (complex_tensor_lanczos.cc:34-56) diagonalises the real
    // form (2 psi_dim) with the one-CTA Jacobi while that fits in shared memory
    // (psi_dim <= 56); above, up to psi_dim 99, its global-memory form takes
    // 50-300 ms a call, so the Krylov run of the same operator takes over: its
    // space is the whole one after psi_dim steps at most, and it stops at the
    // same ground state (any vector of it, if degenerate).
    if (h->site.ket.size < 100 && sym_jacobi_in_shared(2 * (int)h->site.ket.size)) {
        if (iters) *iters = 0;
        return zexact(*h, psi, energy);
    }
    return zkrylov(*h, psi, niter, precision, zero_tol, energy, iters);
}

}  // extern "C"
