// a4/a5: the Lanczos eigensolver of one site step, on the device.
//
// Follows RealTensorLanczos::LanczosMethod (src/dmrg/realdmrg/
// real_tensor_lanczos.cc:14-201):
//   h starts at 0;  per iteration i:  h += H v_i;  alpha_i = <v_i|h>;
//   h -= alpha_i v_i;  beta_i = ||h||;  lowest eigenvalue E_i of the tridiagonal;
//   stop when beta_i < zero_tol, |E_i - E_{i-1}| < precision or i+1 == niter;
//   else v_{i+1} = h / beta_i, h = -beta_i v_i, v_{i+1} orthogonalised against
//   v_0..v_i and normalised;  ground vector = sum_k y_k v_k.
// Differences by design: the reorthogonalisation is classical Gram-Schmidt
// applied twice (two multi-dot/update launch pairs) instead of one modified
// Gram-Schmidt pass (2(i+1) dependent launches); the tridiagonal's lowest
// eigenvalue comes from Sturm bisection on the device instead of dsyevd.
// psi_dim < 100 takes the reference's exact-diagonalisation branch (:34-56):
// the dense H_eff is assembled column by column from matvecs on unit vectors
// and diagonalised by a device Jacobi solver.
// Split-precision operators (DMRG_PREC_TF32X3 / _BF16X3): a first Krylov run with tensor-core
// matvecs, then the FP64 run above from its Ritz vector (FP64 for the dense
// branch, the recurrence, reorthogonalisation, the tridiagonal problem and the
// energy).
#include <atomic>
#include <algorithm>

#include "eig.cuh"
#include "heff.cuh"
#include "vec.cuh"

namespace dmrg {

struct LanczosWork {
    int niter = 0;
    int64_t n = 0;
    DeviceBuffer V, h, scal, state, jac, y, dense, x;
    ReduceScratch rs;
    int* h_state = nullptr;  // the context's pinned words: [done, dim, ...]
    int split_iters = 0;     // Krylov dimension of the last split-precision phase
    // the captured Krylov loop, one per matvec precision (0: FP64, 1: split),
    // with the launch constants it was captured for
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        int niter = 0;
        double precision = 0, zero_tol = 0;
        cudaStream_t stream = nullptr;
    } graph[2];
    ~LanczosWork() {
        for (Graph& g : graph)
            if (g.exec) cudaGraphExecDestroy(g.exec);
    }
};

}  // namespace dmrg

using namespace dmrg;

dmrg_heff_s::~dmrg_heff_s() { delete lw; }

namespace {

// Convergence of the split-precision phase: |E_i - E_{i-1}| below this (the
// matvec's relative error is ~1e-6, the Ritz value settles well before).
constexpr double kSplitPrecision = 1e-9;

// Matvecs of the FP64 run that ends a mixed-precision Lanczos (<= 0: the full
// run to the reference's convergence; dmrg_lanczos_set_polish).
std::atomic<int> g_polish{4};

// End of one captured Lanczos iteration: advance the device's iteration
// counter and keep the loop going while the run has not converged.  The loop is
// bounded: the tridiagonal step marks the run converged at dimension niter.
__global__ void lanczos_advance_kernel(int* state, int niter, cudaGraphConditionalHandle loop) {
    const int it = state[kIterSlot] + 1;
    state[kIterSlot] = it;
    cudaGraphSetConditional(loop, (state[0] == 0 && it < niter) ? 1u : 0u);
}

__global__ void unit_vector_kernel(double* x, int64_t n, int64_t c) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = i == c ? 1.0 : 0.0;
}

// A[r][c] = H[r][c] taken from the upper triangle (the reference diagonalises with
// uplo='U' on the row-major H, general.cc:47-64); cols[c*n + r] = (H e_c)[r].
__global__ void symmetrize_upper_kernel(const double* __restrict__ cols, double* __restrict__ A, int n) {
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n * n; idx += gridDim.x * blockDim.x) {
        const int r = idx / n, c = idx % n;
        A[idx] = r <= c ? cols[(int64_t)c * n + r] : cols[(int64_t)r * n + c];
    }
}

__global__ void column_copy_kernel(const double* __restrict__ Z, int n, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = Z[i * n];
}

int ensure_work(dmrg_heff_s& h, int niter) {
    if (!h.lw) h.lw = new LanczosWork();
    LanczosWork& w = *h.lw;
    const int64_t n = h.site.ket.size;
    if (w.niter < niter || w.n != n) {
        DMRG_TRY(w.V.alloc((size_t)std::max(niter, 1) * std::max<int64_t>(n, 1) * sizeof(double)));
        DMRG_TRY(w.h.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(double)));
        DMRG_TRY(w.scal.alloc((size_t)(4 * std::max(niter, 1) + 16) * sizeof(double)));
        DMRG_TRY(w.y.alloc((size_t)std::max(niter, 1) * sizeof(double)));
        const int m = std::max(niter, 128);
        DMRG_TRY(w.jac.alloc((size_t)(2 * m * m + 4 * m) * sizeof(double)));
        w.niter = niter;
        w.n = n;
    }
    DMRG_TRY(w.x.alloc((size_t)std::max<int64_t>(n, 1) * sizeof(double)));
    DMRG_TRY(w.state.alloc(16 * sizeof(int)));
    DMRG_TRY(w.rs.alloc(std::max(2 * h.ctx->num_sms, 64), std::max(niter, 1)));
    w.h_state = h.ctx->h_pinned;
    return DMRG_OK;
}

int run_exact(dmrg_heff_s& h, double* psi, double* energy) {
    LanczosWork& w = *h.lw;
    const int n = (int)h.site.ket.size;
    cudaStream_t st = h.ctx->stream;
    DMRG_TRY(w.dense.alloc((size_t)(3 * n * n + 4 * n + 8) * sizeof(double)));
    double* cols = w.dense.as<double>();
    double* A = cols + (size_t)n * n;
    double* Z = A + (size_t)n * n;
    double* ev = Z + (size_t)n * n;
    double* e = w.h.as<double>();
    for (int c = 0; c < n; ++c) {
        DMRG_LAUNCH unit_vector_kernel<<<1, 128, 0, st>>>(e, n, c);
        DMRG_TRY(heff_apply_fp64(h, e, cols + (size_t)c * n, false));  // the dense branch stays FP64
    }
    DMRG_LAUNCH symmetrize_upper_kernel<<<std::max(1, (n * n + 255) / 256), 256, 0, st>>>(cols, A, n);
    DMRG_CUDA_TRY(cudaMemsetAsync(w.state.ptr, 0, 16 * sizeof(int), st));
    DMRG_TRY(launch_sym_jacobi(A, n, ev, Z, w.jac.as<double>(), w.state.as<int>() + 2, st));
    DMRG_LAUNCH column_copy_kernel<<<1, 128, 0, st>>>(Z, n, psi);
    double e0 = 0.0;
    DMRG_CUDA_TRY(cudaMemcpyAsync(&e0, ev, sizeof(double), cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaMemcpyAsync(w.h_state, w.state.ptr, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaStreamSynchronize(st));
    if (w.h_state[2] != 0) return set_error(DMRG_E_NUMERIC, "Jacobi eigensolver did not converge (n=%d)", n);
    *energy = e0;
    return DMRG_OK;
}

// One Lanczos iteration i (i read on the device) for the captured loop:
// h += H x;  alpha_i = <x|h>;  h -= alpha_i x;  beta_i = ||h||;  tridiagonal
// step and convergence test;  unless converged: V_{i+1} = h / beta_i, h =
// -beta_i x, reorthogonalised and normalised, x = V_{i+1};  i += 1.  x holds
// V_i (the matvec input) so that the schedules' fixed operand pointers serve
// every iteration.
int capture_iteration(dmrg_heff_s& h, int niter, double precision, double zero_tol, bool split,
                      cudaGraphConditionalHandle loop, cudaStream_t st) {
    LanczosWork& w = *h.lw;
    const int64_t n = h.site.ket.size;
    const int blocks = std::min<int64_t>((n + kVecThreads - 1) / kVecThreads, 2 * h.ctx->num_sms);
    double* V = w.V.as<double>();
    double* hv = w.h.as<double>();
    double* x = w.x.as<double>();
    double* alpha = w.scal.as<double>();
    double* beta = alpha + niter;
    double* E = beta + niter;
    double* c = E + niter;
    double* tmp = c + niter;
    int* state = w.state.as<int>();
    DMRG_TRY(split ? heff_apply_internal(h, x, hv, true) : heff_apply_fp64(h, x, hv, true));
    DMRG_TRY(vec_dot_it(x, hv, n, alpha, state, w.rs, blocks, st));
    DMRG_TRY(vec_axpy_norm_it(alpha, x, hv, n, beta, state, w.rs, blocks, st));
    DMRG_TRY(launch_tridiag_lowest_it(alpha, beta, state + kIterSlot, E, state, precision, zero_tol, niter, st));
    DMRG_TRY(vec_lanczos_step_it(beta, x, hv, V, n, niter, c, tmp, x, state, w.rs, blocks, st));
    DMRG_LAUNCH lanczos_advance_kernel<<<1, 1, 0, st>>>(state, niter, loop);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

// Captures the Krylov loop of one run as a CUDA graph: a conditional WHILE node
// whose body is one iteration (capture_iteration), so a whole Lanczos run is
// one graph launch with no host round trip; the graph is kept and relaunched
// while the operator, niter and the stopping constants stay the same.
int build_loop_graph(dmrg_heff_s& h, int niter, double precision, double zero_tol, bool split) {
    LanczosWork& w = *h.lw;
    LanczosWork::Graph& g = w.graph[split ? 1 : 0];
    cudaStream_t st = h.ctx->stream;
    if (g.exec && g.niter == niter && g.precision == precision && g.zero_tol == zero_tol && g.stream == st)
        return DMRG_OK;
    if (g.exec) {
        cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    DMRG_CUDA_TRY(cudaGraphCreate(&graph, 0));
    int rc = DMRG_OK;
    cudaGraphConditionalHandle loop{};
    cudaError_t e = cudaGraphConditionalHandleCreate(&loop, graph, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams cp{};
    cudaGraphNode_t node = nullptr;
    if (e == cudaSuccess) {
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = loop;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        e = cudaGraphAddNode(&node, graph, nullptr, 0, &cp);
    }
    if (e == cudaSuccess) e = cudaStreamBeginCaptureToGraph(st, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                            cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return set_error(DMRG_E_CUDA, "Lanczos loop graph: %s", cudaGetErrorString(e));
    }
    rc = capture_iteration(h, niter, precision, zero_tol, split, loop, st);
    cudaGraph_t body = nullptr;
    e = cudaStreamEndCapture(st, &body);  // always ends the capture, also after a failed step
    if (rc == DMRG_OK && e != cudaSuccess) rc = set_error(DMRG_E_CUDA, "Lanczos loop capture: %s", cudaGetErrorString(e));
    if (rc == DMRG_OK) {
        e = cudaGraphInstantiate(&g.exec, graph, 0);
        if (e != cudaSuccess) {
            g.exec = nullptr;
            rc = set_error(DMRG_E_CUDA, "Lanczos loop graph instantiation: %s", cudaGetErrorString(e));
        }
    }
    cudaGraphDestroy(graph);
    if (rc != DMRG_OK) return rc;
    g.niter = niter;
    g.precision = precision;
    g.zero_tol = zero_tol;
    g.stream = st;
    return DMRG_OK;
}

// One Lanczos run from psi (real_tensor_lanczos.cc:57-185): matvecs in the
// operator's split precision when `split`, else FP64; vectors, recurrence,
// reorthogonalisation and the tridiagonal problem always FP64.
int krylov(dmrg_heff_s& h, double* psi, int niter, double precision, double zero_tol, bool split, double* energy,
           int* iters) {
    LanczosWork& w = *h.lw;
    const int64_t n = h.site.ket.size;
    cudaStream_t st = h.ctx->stream;
    const int blocks = std::min<int64_t>((n + kVecThreads - 1) / kVecThreads, 2 * h.ctx->num_sms);
    double* V = w.V.as<double>();
    double* hv = w.h.as<double>();
    double* alpha = w.scal.as<double>();
    double* beta = alpha + niter;
    double* E = beta + niter;
    double* c = E + niter;
    double* tmp = c + niter;
    int* state = w.state.as<int>();
    DMRG_CUDA_TRY(cudaMemcpyAsync(V, psi, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    DMRG_CUDA_TRY(cudaMemsetAsync(hv, 0, n * sizeof(double), st));
    DMRG_CUDA_TRY(cudaMemsetAsync(state, 0, 16 * sizeof(int), st));
    int dim = 0;
    if (h.use_graph) {
        // the whole loop as one graph launch; the host reads the result once
        DMRG_TRY(build_loop_graph(h, niter, precision, zero_tol, split));
        DMRG_CUDA_TRY(cudaMemcpyAsync(w.x.ptr, psi, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        DMRG_CUDA_TRY(cudaGraphLaunch(w.graph[split ? 1 : 0].exec, st));
        DMRG_CUDA_TRY(cudaMemcpyAsync(w.h_state, state, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
        DMRG_CUDA_TRY(cudaStreamSynchronize(st));
        dim = w.h_state[0] ? w.h_state[1] : 0;
    }
    // The convergence test runs on the device (tridiag_lowest_kernel records the
    // first dimension that meets it and ignores later calls).  The host reads it
    // once per `chunk` iterations instead of after each one, so the GPU is not
    // left idle between iterations; the few iterations enqueued past
    // convergence write vectors and coefficients beyond `dim`, which nothing
    // reads.  Cheap matvecs get longer chunks.
    const int chunk = (int)std::min<int64_t>(8, std::max<int64_t>(2, 2000000 / (n + 100000)));
    for (int i = 0; i < niter && !h.use_graph; ++i) {
        double* vi = V + (int64_t)i * n;
        DMRG_TRY(split ? heff_apply_internal(h, vi, hv, true) : heff_apply_fp64(h, vi, hv, true));
        DMRG_TRY(vec_dot(vi, hv, n, alpha + i, w.rs, blocks, st));
        DMRG_TRY(vec_axpy_norm(alpha + i, vi, hv, n, beta + i, w.rs, blocks, st));
        DMRG_TRY(launch_tridiag_lowest(alpha, beta, i + 1, E, state, precision, zero_tol, niter, st));
        if ((i + 1) % chunk == 0 || i + 1 == niter) {
            DMRG_CUDA_TRY(cudaMemcpyAsync(w.h_state, state, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
            DMRG_CUDA_TRY(cudaStreamSynchronize(st));
            if (w.h_state[0]) {
                dim = w.h_state[1];
                break;
            }
        }
        if (i + 1 == niter) break;  // the last vector slot is V[niter - 1]
        double* vn = V + (int64_t)(i + 1) * n;
        DMRG_TRY(vec_lanczos_shift(beta + i, vi, hv, vn, n, blocks, st));
        // classical Gram-Schmidt twice; the second pass also normalises
        DMRG_TRY(vec_multidot(V, n, i + 1, vn, n, c, w.rs, blocks, st));
        DMRG_TRY(vec_combine(V, n, i + 1, c, -1.0, vn, 1.0, n, blocks, st));
        DMRG_TRY(vec_multidot(V, n, i + 1, vn, n, c, w.rs, blocks, st));
        DMRG_TRY(vec_combine_normalize(V, n, i + 1, c, -1.0, vn, n, tmp, w.rs, blocks, st));
    }
    if (dim <= 0) return set_error(DMRG_E_NUMERIC, "Lanczos ended without a converged dimension");
    DMRG_TRY(launch_tridiag_ground_vector(alpha, beta, E, state + 1, w.y.as<double>(), state + 2, st));
    DMRG_TRY(vec_combine(V, n, dim, w.y.as<double>(), 1.0, psi, 0.0, n, blocks, st));
    double e = 0.0;
    DMRG_CUDA_TRY(cudaMemcpyAsync(&e, E + dim - 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaMemcpyAsync(w.h_state, state, 4 * sizeof(int), cudaMemcpyDeviceToHost, st));
    DMRG_CUDA_TRY(cudaStreamSynchronize(st));
    if (w.h_state[2] != 0) return set_error(DMRG_E_NUMERIC, "tridiagonal ground vector failed (m=%d)", dim);
    if (split) DMRG_TRY(take_device_status(h.ctx));  // a tensor-core wait that gave up
    *energy = e;
    if (iters) *iters = dim;
    return DMRG_OK;
}

}  // namespace

extern "C" int dmrg_heff_set_graph(dmrg_heff_t h, int enable) {
    if (!h) return set_error(DMRG_E_ARG, "null operator");
    h->use_graph = enable != 0;
    return DMRG_OK;
}

extern "C" int dmrg_lanczos_set_polish(int iters) {
    g_polish.store(iters);
    return DMRG_OK;
}

extern "C" int dmrg_heff_set_split_threshold(dmrg_heff_t h, int64_t min_psi_dim) {
    if (!h || min_psi_dim < 0) return set_error(DMRG_E_ARG, "invalid split threshold");
    h->split_min_dim = min_psi_dim;
    return DMRG_OK;
}

extern "C" int dmrg_heff_split_iters(dmrg_heff_t h, int* iters) {
    if (!h || !iters) return set_error(DMRG_E_ARG, "null argument");
    *iters = h->lw ? h->lw->split_iters : 0;
    return DMRG_OK;
}

extern "C" int dmrg_lanczos(dmrg_heff_t hp, double* psi, int niter, double precision, double zero_tol,
                            double* energy, int* iters) {
    if (!hp || !psi || !energy || niter <= 0) return set_error(DMRG_E_ARG, "invalid Lanczos arguments");
    if (niter > kMaxVec) return set_error(DMRG_E_ARG, "niter %d above %d", niter, kMaxVec);
    dmrg_heff_s& h = *hp;
    DMRG_TRY(ensure_work(h, niter));
    const int64_t n = h.site.ket.size;
    if (n < 100) {  // exact diagonalisation branch (real_tensor_lanczos.cc:34)
        if (iters) *iters = 0;
        return run_exact(h, psi, energy);
    }
    // A split Krylov phase pays off only where the split matvec is clearly faster
    // than the FP64 one (large blocks); below h.split_min_dim the FP64 run alone
    // is cheaper than the two phases.
    if (!is_split(h.precision) || n < h.split_min_dim) {
        h.lw->split_iters = 0;
        return krylov(h, psi, niter, precision, zero_tol, false, energy, iters);
    }
    // Mixed precision: a Krylov run on split-precision matvecs until the Ritz
    // value settles at the split arithmetic's resolution, then an FP64 Krylov
    // run from that Ritz vector: a short one of g_polish matvecs (its lowest
    // Ritz value is the energy, with an error quadratic in the split vector's,
    // and its Ritz vector the state), or with g_polish <= 0 the reference's
    // full run to its own convergence.
    double e_split = 0.0;
    int it_split = 0;
    DMRG_TRY(krylov(h, psi, niter, kSplitPrecision, zero_tol, true, &e_split, &it_split));
    LanczosWork& w = *h.lw;
    const int blocks = (int)std::min<int64_t>((n + kVecThreads - 1) / kVecThreads, 2 * h.ctx->num_sms);
    DMRG_TRY(vec_normalize(psi, n, w.scal.as<double>() + 4 * niter, w.rs, blocks, h.ctx->stream));
    int it_fp64 = 0;
    const int polish = g_polish.load();
    DMRG_TRY(krylov(h, psi, polish > 0 ? std::min(polish, niter) : niter, precision, zero_tol, false, energy,
                    &it_fp64));
    w.split_iters = it_split;
    if (iters) *iters = it_fp64;
    return DMRG_OK;
}
