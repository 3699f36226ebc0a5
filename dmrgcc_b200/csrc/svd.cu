// Batched one-sided block-Jacobi SVD (see svd.cuh).
#include <atomic>
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "svd.cuh"

namespace dmrg {
namespace {

constexpr int kBlk = 32;        // columns per block
constexpr int kPair = 64;       // columns per pair
constexpr int kChunk = 32;      // rows per streamed chunk
#ifndef DMRG_SVD_SOLVE_THREADS
#define DMRG_SVD_SOLVE_THREADS 512
#endif
constexpr int kThreads = DMRG_SVD_SOLVE_THREADS;   // pair-solve CTA
constexpr int kLd = kPair + 1;  // padded row of the shared 64x64 matrices
#ifndef DMRG_SVD_INNER_SWEEPS
#define DMRG_SVD_INNER_SWEEPS 2
#endif
constexpr int kInnerSweeps = DMRG_SVD_INNER_SWEEPS;
constexpr int kMaxSweeps = 40;
// The sweep cap in force (dmrg_svd_set_max_sweeps lowers it to provoke the
// did-not-converge path without touching the device).
std::atomic<int> g_max_sweeps{kMaxSweeps};
#ifndef DMRG_SVD_GRAM_MIN_ROWS
#define DMRG_SVD_GRAM_MIN_ROWS 64
#endif
constexpr int kGramMinRows = DMRG_SVD_GRAM_MIN_ROWS;  // rows of a Gram item, at least (multiple of 32)
// Columns whose norm is below kZeroRel * sqrt(rows) * ||A||_F are rounding
// residue of a rank-deficient matrix: they take part in no rotation and in no
// convergence test (their values are below any truncation threshold that is
// meaningful in FP64; rotating them only stirs rounding noise).
constexpr double kZeroRel = 4.0 * DBL_EPSILON;

constexpr int kSteps = kPair - 1;                 // steps of one cyclic sweep of a pair
constexpr int kMaxSteps = kInnerSweeps * kSteps;  // rotation log capacity

struct SvdSmem {
    // the Gram matrix, double-buffered: a step reads one copy and writes the
    // other, so that one barrier per step orders every read before the writes
    double G[2][kPair * kLd];
    // rotation log: step t, seat lane j -> (c, s) of the rotation of the two
    // columns seated at lane j (see seat_column), oriented (first, second)
    double2 log[kMaxSteps * (kPair / 2)];
    double2 cs[kPair / 2];   // (c, s) of the step's rotation k, oriented as schedule entry k addresses it
    int active[2];           // by step parity: the step rotates something
    double red[kThreads / 32];
    double flag;
    uint32_t sched[kSteps * (kPair / 2)];   // the pair schedule (pair_schedule())
};

// Seating of the pair solve's columns (the circle method of a round-robin
// tournament): at step r, seat 0 holds column 0 and seat s >= 1 holds column
// ((s - 1 - r) mod 63) + 1; seat lane j owns seats j and 63 - j, whose columns
// are the pair rotated at that step.  From one step to the next the column in
// seat s moves to seat s + 1 (seat 63 to seat 1; seat 0 stays), so a lane's two
// columns reach their next seats by one shuffle each way.
__host__ __device__ __forceinline__ int seat_column(int seat, int r) {
    return seat == 0 ? 0 : ((seat - 1 - r) % kSteps + kSteps) % kSteps + 1;
}

__host__ __device__ __forceinline__ void rr_pair(int r, int i, int N, int& p, int& q) {
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

__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Stage 1 of a round: partial Gram matrices.  Item = (pair task, row range of W);
// 128 threads (2x2 warps, 32x32 each = 4x4 DMMA tiles); G_part = X^T X over the
// item's rows, X = the pair's 64 columns, streamed 32 rows at a time into a
// column-major shared tile (row pad 4: conflict-free stores and fragment reads).
constexpr int kGramLd = kChunk + 4;
__global__ void __launch_bounds__(128) gram_kernel(const SvdProblem* __restrict__ probs,
                                                   const SvdTask* __restrict__ tasks,
                                                   const SvdItem* __restrict__ items,
                                                   const int* __restrict__ colmap, const double* __restrict__ W,
                                                   double* __restrict__ gpart) {
    __shared__ double Xt[kPair * kGramLd];  // Xt[c][k]
    const SvdItem it = items[blockIdx.x];
    const SvdTask task = tasks[it.task];
    const SvdProblem p = probs[task.problem];
    const int colI = task.bi * kBlk, colJ = task.bj * kBlk;
    const double* Wp = W + p.w_off;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp >> 1, wn = warp & 1, fr = lane >> 2, fc = lane & 3;
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    // thread: row k of each chunk in columns c = warp + 4e (e < 16); the column
    // offsets are looked up once, and the next chunk is loaded into registers
    // while the tensor cores work on the current one
    constexpr int kCols = kChunk * kPair / 128;
    static_assert(kChunk == 32 && kCols * 128 == kChunk * kPair, "one row per lane");
    const int k = lane;
    int64_t coff[kCols];
#pragma unroll
    for (int e = 0; e < kCols; ++e) {
        const int c = warp + 4 * e;
        const int vc = c < kBlk ? colI + c : colJ + c - kBlk;
        coff[e] = vc < p.cols ? (int64_t)colmap[p.perm_off + vc] * p.rows : -1;
    }
    double nxt[kCols];
#pragma unroll
    for (int e = 0; e < kCols; ++e) nxt[e] = (coff[e] >= 0 && it.r0 + k < it.r1) ? Wp[coff[e] + it.r0 + k] : 0.0;
    for (int k0 = it.r0; k0 < it.r1; k0 += kChunk) {
#pragma unroll
        for (int e = 0; e < kCols; ++e) Xt[(warp + 4 * e) * kGramLd + k] = nxt[e];
        __syncthreads();
        const int k1 = k0 + kChunk;
        if (k1 < it.r1) {
#pragma unroll
            for (int e = 0; e < kCols; ++e) nxt[e] = (coff[e] >= 0 && k1 + k < it.r1) ? Wp[coff[e] + k1 + k] : 0.0;
        }
#pragma unroll
        for (int kk = 0; kk < kChunk; kk += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = Xt[(wm * 32 + i * 8 + fr) * kGramLd + kk + fc];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Xt[(wn * 32 + j * 8 + fr) * kGramLd + kk + fc];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
        __syncthreads();
    }
    double* g = gpart + (int64_t)blockIdx.x * kPair * kPair;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int row = wm * 32 + i * 8 + fr, col = wn * 32 + j * 8 + 2 * fc;
            g[row * kPair + col] = acc[i][j][0];
            g[row * kPair + col + 1] = acc[i][j][1];
        }
}

// Convergence measure of a sweep: one CTA per tile (problem, bi <= bj), the
// 32x32 block X_bi^T X_bj of the sector's Gram matrix over all rows (DMMA, 2x2
// warps of 16x16), reduced to the largest pair measure
// |g_ab| / (||A||_F max(|x_a|, |x_b|)) over its column pairs a < b (norms from
// the sweep's column norms), skipping columns at rounding level.
__global__ void __launch_bounds__(128) measure_kernel(const SvdProblem* __restrict__ probs,
                                                      const SvdTile* __restrict__ tiles,
                                                      const int* __restrict__ colmap, const double* __restrict__ W,
                                                      const double* __restrict__ norm, const double* __restrict__ fro2,
                                                      double* __restrict__ bm) {
    __shared__ double Xt[kPair * kGramLd];  // Xt[c][k]: c < 32 block bi, c >= 32 block bj
    __shared__ double red[4];
    const SvdTile tile = tiles[blockIdx.x];
    const SvdProblem p = probs[tile.problem];
    const int colI = tile.bi * kBlk, colJ = tile.bj * kBlk;
    const double* Wp = W + p.w_off;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp >> 1, wn = warp & 1, fr = lane >> 2, fc = lane & 3;
    double acc[2][2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    constexpr int kCols = kChunk * kPair / 128;
    const int k = lane;
    int64_t coff[kCols];
#pragma unroll
    for (int e = 0; e < kCols; ++e) {
        const int c = warp + 4 * e;
        const int vc = c < kBlk ? colI + c : colJ + c - kBlk;
        coff[e] = vc < p.cols ? (int64_t)colmap[p.perm_off + vc] * p.rows : -1;
    }
    double nxt[kCols];
#pragma unroll
    for (int e = 0; e < kCols; ++e) nxt[e] = (coff[e] >= 0 && k < p.rows) ? Wp[coff[e] + k] : 0.0;
    for (int k0 = 0; k0 < p.rows; k0 += kChunk) {
#pragma unroll
        for (int e = 0; e < kCols; ++e) Xt[(warp + 4 * e) * kGramLd + k] = nxt[e];
        __syncthreads();
        const int k1 = k0 + kChunk;
        if (k1 < p.rows) {
#pragma unroll
            for (int e = 0; e < kCols; ++e) nxt[e] = (coff[e] >= 0 && k1 + k < p.rows) ? Wp[coff[e] + k1 + k] : 0.0;
        }
#pragma unroll
        for (int kk = 0; kk < kChunk; kk += 4) {
            double a[2], b[2];
#pragma unroll
            for (int i = 0; i < 2; ++i) a[i] = Xt[(wm * 16 + i * 8 + fr) * kGramLd + kk + fc];
#pragma unroll
            for (int j = 0; j < 2; ++j) b[j] = Xt[(kBlk + wn * 16 + j * 8 + fr) * kGramLd + kk + fc];
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
        __syncthreads();
    }
    const double f2 = fro2[tile.problem];
    const double fro = sqrt(f2);
    const double zero2 = kZeroRel * kZeroRel * (double)p.rows * f2;
    double worst = 0.0;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int a = colI + wm * 16 + i * 8 + fr, b = colJ + wn * 16 + j * 8 + 2 * fc + h;
                if (a >= p.cols || b >= p.cols || a >= b) continue;
                const double na = norm[p.s_off + colmap[p.perm_off + a]], nb = norm[p.s_off + colmap[p.perm_off + b]];
                if (na * na <= zero2 || nb * nb <= zero2) continue;
                worst = fmax(worst, fabs(acc[i][j][h]) / (fro * fmax(na, nb)));
            }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) worst = fmax(worst, __shfl_xor_sync(0xffffffffu, worst, o));
    if (lane == 0) red[warp] = worst;
    __syncthreads();
    if (threadIdx.x == 0) bm[blockIdx.x] = fmax(fmax(red[0], red[1]), fmax(red[2], red[3]));
}

// Stage 2: one CTA per pair task.  Sums the task's partial Gram matrices (fixed
// order), measures the pair's convergence, and (unless converged) runs a few
// cyclic Jacobi sweeps on the 64x64 Gram matrix, writing the accumulated 64x64
// rotation to rot[task - first] and skip[task - first] = 0.
__global__ void __launch_bounds__(kThreads) solve_kernel(const SvdProblem* __restrict__ probs,
                                                         const SvdTask* __restrict__ tasks, int first,
                                                         const double* __restrict__ gpart,
                                                         const double* __restrict__ fro2, double* __restrict__ rot,
                                                         int* __restrict__ skip, const uint32_t* __restrict__ sched,
                                                         int inner_sweeps) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SvdSmem& S = *reinterpret_cast<SvdSmem*>(smem_raw);
    const int t = first + blockIdx.x;
    const SvdTask task = tasks[t];
    const SvdProblem p = probs[task.problem];
    const double tol = 2.0 * DBL_EPSILON * sqrt((double)p.rows);
    const double zero2 = kZeroRel * kZeroRel * (double)p.rows * fro2[task.problem];
    {
        // the partials in a fixed order (c ascending) per entry; the entries of
        // a thread are independent, so all of a partial's loads are in flight
        constexpr int kElems = kPair * kPair / kThreads;
        static_assert(kPair * kPair % kThreads == 0, "even split");
        double v[kElems];
#pragma unroll
        for (int u = 0; u < kElems; ++u) v[u] = 0.0;
        const double* gp = gpart + (int64_t)task.g_first * kPair * kPair + threadIdx.x;
        for (int c = 0; c < task.g_count; ++c, gp += kPair * kPair)
#pragma unroll
            for (int u = 0; u < kElems; ++u) v[u] += gp[u * kThreads];
#pragma unroll
        for (int u = 0; u < kElems; ++u) {
            const int idx = threadIdx.x + u * kThreads;
            S.G[0][(idx / kPair) * kLd + idx % kPair] = v[u];
        }
    }
    for (int idx = threadIdx.x; idx < kSteps * (kPair / 2); idx += kThreads) S.sched[idx] = sched[idx];
    __syncthreads();

    // ---- convergence measure over the pair: |g_ij| / (||A||_F max(|x_i|, |x_j|)),
    // the size (relative to ||A||_F) of the perturbation of A that leaving the pair
    // unrotated amounts to.  Below tol the pair is as converged as a backward
    // stable SVD can tell (for two columns of norm ~||A|| this is the usual
    // relative test; a column far below ||A|| needs only an angle ~tol ||A|| / |x|).
    const double fro = sqrt(fro2[task.problem]);
    double worst = 0.0;
    for (int idx = threadIdx.x; idx < kPair * kPair; idx += kThreads) {
        const int a = idx / kPair, b = idx % kPair;
        if (a >= b) continue;
        const double ga = S.G[0][a * kLd + a], gb = S.G[0][b * kLd + b];
        if (ga > zero2 && gb > zero2) worst = fmax(worst, fabs(S.G[0][a * kLd + b]) / (fro * sqrt(fmax(ga, gb))));
    }
    worst = block_max(worst, S);
    if (threadIdx.x == 0) skip[blockIdx.x] = worst <= tol ? 1 : 0;
    if (worst <= tol) return;  // pair already orthogonal: nothing to rotate

    // A pair whose off-diagonal measure is at or below tol needs no rotation (the
    // same test decides convergence); a step that rotates nothing skips the
    // update, and the solve ends once a sweep leaves every measure at or below tol.
    // rotation test: |g_ab| above half the convergence threshold, so that every
    // pair the measure above calls unconverged is rotated whatever the rounding
    // of either expression
    const double tol2f = 0.25 * tol * tol * fro * fro;
    constexpr int kWarps = kThreads / 32;
    constexpr int kItems = (kPair / 2) * (kPair / 2) / kThreads;  // 2x2 Gram blocks per thread
    constexpr int kQRows = kPair / kWarps;                         // rows of Q per warp
    static_assert(kThreads % 32 == 0 && kItems * kThreads == (kPair / 2) * (kPair / 2) && kQRows * kWarps == kPair,
                  "even split of the Gram blocks and of the rows of Q");
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int steps = 0;  // rotation log entries written
    int cur = 0;    // the copy of G holding the current matrix
    for (int sweep = 0; sweep < inner_sweeps; ++sweep) {
        bool rotated = false;
        for (int r = 0; r < kSteps; ++r, ++steps) {
            // Warp 0 computes the step's 32 rotations (lane k: the pair of schedule
            // entry k) while the other warps load the entries they update (the
            // addresses come from the static schedule); a barrier publishes the
            // rotations, and a step that rotates nothing ends there.
            const unsigned e = S.sched[r * (kPair / 2) + lane];
            const int pc = (e >> 12) & 1 ? (e >> 6) & 63 : e & 63;  // the lane's columns in the order it addresses them
            const int qc = (e >> 12) & 1 ? e & 63 : (e >> 6) & 63;
            const double* Gc = S.G[cur];
            int pi[kItems], qi[kItems];
            double x[kItems][4];
#pragma unroll
            for (int u = 0; u < kItems; ++u) {
                const unsigned ei = S.sched[r * (kPair / 2) + warp + kWarps * u];  // the row pair's entry
                pi[u] = (ei >> 12) & 1 ? (ei >> 6) & 63 : ei & 63;
                qi[u] = (ei >> 12) & 1 ? ei & 63 : (ei >> 6) & 63;
                x[u][0] = Gc[pi[u] * kLd + pc];
                x[u][1] = Gc[pi[u] * kLd + qc];
                x[u][2] = Gc[qi[u] * kLd + pc];
                x[u][3] = Gc[qi[u] * kLd + qc];
            }
            if (warp == 0) {
                const int a = e & 63, b = (e >> 6) & 63;  // a < b
                const double apq = Gc[a * kLd + b];
                const double daa = Gc[a * kLd + a], dbb = Gc[b * kLd + b];
                double c = 1.0, s = 0.0;
                if (daa > zero2 && dbb > zero2 && apq * apq > tol2f * fmax(daa, dbb)) {
                    // The rotation with tan = sign(x) y / (|x| + sqrt(x^2 + y^2)),
                    // x = dbb - daa, y = 2 apq (the smaller root of the Jacobi
                    // equation), as c = u / sqrt(u^2 + y^2), s = sign(x) y / sqrt(u^2 + y^2)
                    // with u = |x| + sqrt(x^2 + y^2): no division.
                    const double xd = dbb - daa, y = 2.0 * apq;
                    const double u = fabs(xd) + sqrt(xd * xd + y * y);
                    const double rn = rsqrt(u * u + y * y);
                    c = u * rn;
                    s = (xd >= 0.0 ? y : -y) * rn;
                }
                // the lane addresses p first: rotating (b, a) by (c, -s) is rotating (a, b) by (c, s)
                const double se = (e >> 12) & 1 ? -s : s;
                S.cs[lane] = make_double2(c, se);
                S.log[steps * (kPair / 2) + ((e >> 13) & 31)] = make_double2(c, ((e >> 18) & 1) ? -se : se);
                const bool any = __any_sync(0xffffffffu, s != 0.0);
                if (lane == 0) S.active[steps & 1] = any ? 1 : 0;
            }
            __syncthreads();
            if (!S.active[steps & 1]) continue;  // the same verdict for every thread
            rotated = true;
            // G <- J^T G J into the other copy: thread (i, j = lane) takes the 2x2
            // block of rows (p_i, q_i) and columns (p_j, q_j), both rotations at
            // once (an untouched block is copied), for i = warp + kWarps u
            double* Gn = S.G[cur ^ 1];
            const double2 csj = S.cs[lane];
#pragma unroll
            for (int u = 0; u < kItems; ++u) {
                const double2 csi = S.cs[warp + kWarps * u];
                const double ci = csi.x, si = csi.y, c = csj.x, se = csj.y;
                const double y11 = ci * x[u][0] - si * x[u][2], y12 = ci * x[u][1] - si * x[u][3];
                const double y21 = si * x[u][0] + ci * x[u][2], y22 = si * x[u][1] + ci * x[u][3];
                Gn[pi[u] * kLd + pc] = c * y11 - se * y12;
                Gn[pi[u] * kLd + qc] = se * y11 + c * y12;
                Gn[qi[u] * kLd + pc] = c * y21 - se * y22;
                Gn[qi[u] * kLd + qc] = se * y21 + c * y22;
            }
            cur ^= 1;
            __syncthreads();
        }
        if (!rotated || sweep + 1 == inner_sweeps) break;  // uniform: every thread saw the same flags
        // the pair's measure after this sweep: a further sweep only if some entry is above tol
        double off = 0.0;
        for (int idx = threadIdx.x; idx < kPair * kPair; idx += kThreads) {
            const int a = idx / kPair, b = idx % kPair;
            if (a >= b) continue;
            const double ga = S.G[cur][a * kLd + a], gb = S.G[cur][b * kLd + b], g = S.G[cur][a * kLd + b];
            if (ga > zero2 && gb > zero2 && g * g > tol2f * fmax(ga, gb)) off = 1.0;
        }
        if (block_max(off, S) == 0.0) break;
    }
    __syncthreads();  // the log is complete

    // The accumulated rotation Q = J_0 J_1 ... from the log, in registers: warp w
    // takes rows kQRows w ... of Q, lane j the two entries of each row in the
    // columns seated at lane j.  After each step's rotation the entries move to their next
    // seats (seat_column): seat s -> s + 1 for 1 <= s <= 62, seat 63 -> seat 1.
    double q1[kQRows], q2[kQRows];
#pragma unroll
    for (int k = 0; k < kQRows; ++k) {
        const int row = kQRows * warp + k;
        q1[k] = row == lane ? 1.0 : 0.0;               // seat lane (column lane at step 0)
        q2[k] = row == kPair - 1 - lane ? 1.0 : 0.0;   // seat 63 - lane
    }
    for (int t = 0; t < steps; ++t) {
        const double2 cs = S.log[t * (kPair / 2) + lane];
#pragma unroll
        for (int k = 0; k < kQRows; ++k) {
            const double f = cs.x * q1[k] - cs.y * q2[k], g = cs.y * q1[k] + cs.x * q2[k];
            const double up = __shfl_up_sync(0xffffffffu, lane == 0 ? g : f, 1);  // seat j - 1 (lane 0: seat 63)
            const double dn = __shfl_down_sync(0xffffffffu, g, 1);               // seat 62 - j
            q1[k] = lane == 0 ? f : up;
            q2[k] = lane == 31 ? f : dn;
        }
    }
    double* R = rot + (int64_t)blockIdx.x * kPair * kPair;
    const int c1 = seat_column(lane, steps), c2 = seat_column(kPair - 1 - lane, steps);
#pragma unroll
    for (int k = 0; k < kQRows; ++k) {
        const int row = kQRows * warp + k;
        R[row * kPair + c1] = q1[k];
        R[row * kPair + c2] = q2[k];
    }
}

// Stage 3: item = (pair task, segment, row range): the pair's 64 columns of W
// (segment 0) or of the accumulated rotation (segment 1), rows [r0, r1) with
// r1 - r0 <= 64, are multiplied by the task's 64x64 rotation (DMMA, in place).
// Shared tiles: Xt[c][row] and R[c][col], row pad 4 (conflict-free).
constexpr int kRotLd = kPair + 4;
constexpr size_t kRotSmem = 2 * sizeof(double) * kPair * kRotLd;
__global__ void __launch_bounds__(128) rotate_kernel(const SvdProblem* __restrict__ probs,
                                                     const SvdTask* __restrict__ tasks,
                                                     const SvdItem* __restrict__ items, int first,
                                                     const double* __restrict__ rot, const int* __restrict__ skip,
                                                     const int* __restrict__ colmap, double* __restrict__ W,
                                                     double* __restrict__ Qacc) {
    extern __shared__ __align__(16) double rsm[];
    double* Xt = rsm;                   // [64 cols][kRotLd]
    double* R = rsm + kPair * kRotLd;   // [64][kRotLd]
    const SvdItem it = items[blockIdx.x];
    if (skip[it.task - first]) return;
    const SvdTask task = tasks[it.task];
    const SvdProblem p = probs[task.problem];
    const int colI = task.bi * kBlk, colJ = task.bj * kBlk;
    double* base = it.seg == 0 ? W + p.w_off : Qacc + p.q_off;
    const int ld = it.seg == 0 ? p.rows : p.cols;
    const double* Rg = rot + (int64_t)(it.task - first) * kPair * kPair;
    for (int idx = threadIdx.x; idx < kPair * kPair; idx += 128) {
        const int c = idx / kPair, k = idx % kPair;  // consecutive threads: consecutive rows of a column
        const int vc = c < kBlk ? colI + c : colJ + c - kBlk;
        const bool v = vc < p.cols && it.r0 + k < it.r1;
        Xt[c * kRotLd + k] = v ? base[(int64_t)colmap[p.perm_off + vc] * ld + it.r0 + k] : 0.0;
        R[c * kRotLd + k] = Rg[idx];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp >> 1, wn = warp & 1, fr = lane >> 2, fc = lane & 3;
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll 4
    for (int kk = 0; kk < kPair; kk += 4) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = Xt[(kk + fc) * kRotLd + wm * 32 + i * 8 + fr];  // X[row][c]
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = R[(kk + fc) * kRotLd + wn * 32 + j * 8 + fr];   // R[c][col]
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int row = wm * 32 + i * 8 + fr, col = wn * 32 + j * 8 + 2 * fc;
            Xt[col * kRotLd + row] = acc[i][j][0];
            Xt[(col + 1) * kRotLd + row] = acc[i][j][1];
        }
    __syncthreads();
    for (int idx = threadIdx.x; idx < kPair * kPair; idx += 128) {
        const int c = idx / kPair, k = idx % kPair;
        const int vc = c < kBlk ? colI + c : colJ + c - kBlk;
        if (vc < p.cols && it.r0 + k < it.r1) base[(int64_t)colmap[p.perm_off + vc] * ld + it.r0 + k] = Xt[c * kRotLd + k];
    }
}

// Scales each working matrix whose largest magnitude is below 1/2 by the power
// of two that brings it into [0.5, 1), and records the exponent e (0: left
// as is).  Only exponents change, so the scaling is exact; the Gram matrices,
// thresholds and rotations then never meet underflow, however small the
// sector's values (a sector that carries a negligible weight of the state
// reaches 1e-100 and below, whose squares underflow).  unscale_kernel undoes
// it on the result.  Three kernels over grid (problems, kSlices): the slices'
// largest magnitudes; the scaling (each slice takes the problem's maximum over
// the slice maxima) with the slices' sums of squares; the squared Frobenius
// norms, summing the slices in a fixed order.
constexpr int kSlices = 32;
__device__ __forceinline__ void slice_range(int64_t cnt, int slice, int64_t& b, int64_t& e) {
    b = cnt * slice / kSlices;
    e = cnt * (slice + 1) / kSlices;
}

__device__ __forceinline__ double block_reduce(double v, bool take_max) {
    __shared__ double red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double u = __shfl_xor_sync(0xffffffffu, v, o);
        v = take_max ? fmax(v, u) : v + u;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double r = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r = take_max ? fmax(r, red[k]) : r + red[k];
    return r;
}

__global__ void __launch_bounds__(256) slice_max_kernel(const SvdProblem* __restrict__ probs,
                                                        const double* __restrict__ W, double* __restrict__ part) {
    const SvdProblem p = probs[blockIdx.x];
    const double* w = W + p.w_off;
    int64_t b, e;
    slice_range((int64_t)p.rows * p.cols, blockIdx.y, b, e);
    double mx = 0.0;
    for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) mx = fmax(mx, fabs(w[i]));
    mx = block_reduce(mx, true);
    if (threadIdx.x == 0) part[blockIdx.x * kSlices + blockIdx.y] = mx;
}

__global__ void __launch_bounds__(256) prescale_kernel(const SvdProblem* __restrict__ probs, double* __restrict__ W,
                                                       const double* __restrict__ part_max, int* __restrict__ expo,
                                                       double* __restrict__ part_ss) {
    const SvdProblem p = probs[blockIdx.x];
    double m = 0.0;
    for (int k = 0; k < kSlices; ++k) m = fmax(m, part_max[blockIdx.x * kSlices + k]);
    int ex = 0;
    if (m > 0.0 && m < 0.5) frexp(m, &ex);  // m = f 2^e, f in [0.5, 1), e <= -1
    if (blockIdx.y == 0 && threadIdx.x == 0) expo[blockIdx.x] = ex;
    double* w = W + p.w_off;
    int64_t b, e;
    slice_range((int64_t)p.rows * p.cols, blockIdx.y, b, e);
    double ss = 0.0;
    for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) {
        const double v = ex ? ldexp(w[i], -ex) : w[i];
        if (ex) w[i] = v;
        ss += v * v;
    }
    ss = block_reduce(ss, false);
    if (threadIdx.x == 0) part_ss[blockIdx.x * kSlices + blockIdx.y] = ss;
}

// Undoes prescale_kernel on the final working matrix and the sorted singular
// values.  Grid (problems, slices).
__global__ void __launch_bounds__(256) unscale_kernel(const SvdProblem* __restrict__ probs, const int* __restrict__ expo,
                                                      double* __restrict__ W, double* __restrict__ sig) {
    const SvdProblem p = probs[blockIdx.x];
    const int e = expo[blockIdx.x];
    if (e == 0) return;
    double* w = W + p.w_off;
    const int64_t cnt = (int64_t)p.rows * p.cols;
    for (int64_t i = (int64_t)blockIdx.y * blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.y * blockDim.x)
        w[i] = ldexp(w[i], e);
    if (blockIdx.y == 0)
        for (int j = threadIdx.x; j < p.cols; j += blockDim.x) sig[p.s_off + j] = ldexp(sig[p.s_off + j], e);
}

// Squared Frobenius norm of each working matrix: its slices' sums in order.
__global__ void fro2_kernel(const double* __restrict__ part_ss, int np, double* __restrict__ fro2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    double s = 0.0;
    for (int k = 0; k < kSlices; ++k) s += part_ss[i * kSlices + k];
    fro2[i] = s;
}

// Q <- I for every problem.  Grid (problems, kSlices).
__global__ void __launch_bounds__(256) init_identity_kernel(const SvdProblem* __restrict__ probs, double* __restrict__ Q) {
    const SvdProblem p = probs[blockIdx.x];
    double* q = Q + p.q_off;
    int64_t b, e;
    slice_range((int64_t)p.cols * p.cols, blockIdx.y, b, e);
    for (int64_t idx = b + threadIdx.x; idx < e; idx += blockDim.x) q[idx] = (idx / p.cols == idx % p.cols) ? 1.0 : 0.0;
}

// Column norms of every working matrix, one warp per column (fixed reduction order).
__global__ void __launch_bounds__(256) colnorm_kernel(const SvdProblem* __restrict__ probs,
                                                      const double* __restrict__ W, double* __restrict__ norm) {
    const SvdProblem p = probs[blockIdx.x];
    const int lane = threadIdx.x & 31;
    const int j = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (j >= p.cols) return;
    const double* col = W + p.w_off + (int64_t)j * p.rows;
    double s = 0.0;
    for (int k = lane; k < p.rows; k += 32) s += col[k] * col[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) norm[p.s_off + j] = sqrt(s);
}

// Descending order of the column norms (ties by column index): order[rank] = column;
// with `sig`, also the sorted values.  Grid (problems, column slices of 256).
__global__ void __launch_bounds__(256) rank_kernel(const SvdProblem* __restrict__ probs,
                                                   const double* __restrict__ norm, int* __restrict__ order,
                                                   double* __restrict__ sig) {
    const SvdProblem p = probs[blockIdx.x];
    const double* t = norm + p.s_off;
    for (int j = blockIdx.y * blockDim.x + threadIdx.x; j < p.cols; j += gridDim.y * blockDim.x) {
        const double v = t[j];
        int rank = 0;
        for (int o = 0; o < p.cols; ++o) {
            const double u = t[o];
            rank += (u > v) || (u == v && o < j);
        }
        order[p.perm_off + rank] = j;
        if (sig) sig[p.s_off + rank] = v;
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

// Lane order of the pair solve's rotations.  Step r rotates the 32 column pairs
// seated at the 32 seat lanes (seat_column); chosen here is which lane of the
// Gram update takes which pair and which of its two columns the lane addresses
// first.  Entry (r, lane) = a | b << 6 | flip << 12 | j << 13 | jflip << 18:
// a < b the pair's columns, flip = the lane addresses b first, j = the pair's
// seat lane, jflip = the column in seat j is not the one addressed first.
// In each half-warp the 16 first columns lie in 16 distinct 8-byte shared-memory
// banks (column mod 16), and so do the 16 second columns, so that every 8-byte
// access of a step's update takes the minimum of two wavefronts.  Such an order
// always exists: a step's pairs are the edges of a 4-regular multigraph on the 16
// residues; orienting it along closed trails gives each residue in- and
// out-degree 2, and the oriented edges split into two perfect matchings (tail
// residue -> head residue), one per half-warp.  Returns DMRG_OK or, if a check
// of the result fails, DMRG_E_STATE.
int build_pair_schedule(std::vector<uint32_t>& tab) {
    constexpr int kP = kPair / 2, kR = 16;
    tab.assign(kSteps * kP, 0);
    std::vector<int> met(kPair * kPair, 0);
    for (int r = 0; r < kSteps; ++r) {
        int pa[kP], pb[kP], first[kP], tail[kP], head[kP], side[kP];
        bool used[kP];
        std::vector<int> adj[kR];
        for (int k = 0; k < kP; ++k) {
            const int c0 = seat_column(k, r), c1 = seat_column(kPair - 1 - k, r);
            pa[k] = std::min(c0, c1);
            pb[k] = std::max(c0, c1);
            adj[pa[k] % kR].push_back(k);
            adj[pb[k] % kR].push_back(k);
            used[k] = false;
            side[k] = -1;
        }
        // closed trails: from v0, leave each residue along an unused edge; with
        // even degrees the walk can only stop back at v0
        for (int v0 = 0; v0 < kR; ++v0) {
            for (;;) {
                int cur = v0, len = 0;
                for (;;) {
                    int e = -1;
                    for (int x : adj[cur])
                        if (!used[x]) {
                            e = x;
                            break;
                        }
                    if (e < 0) break;
                    used[e] = true;
                    ++len;
                    const bool from_a = pa[e] % kR == cur;
                    first[e] = from_a ? pa[e] : pb[e];
                    tail[e] = cur;
                    head[e] = (from_a ? pb[e] : pa[e]) % kR;
                    cur = head[e];
                }
                if (len == 0) break;
                if (cur != v0) return set_error(DMRG_E_STATE, "pair schedule: open trail");
            }
        }
        // alternate the edges around each cycle of the 2-regular bipartite graph
        for (int e0 = 0; e0 < kP; ++e0) {
            for (int e = e0; side[e] < 0;) {
                side[e] = 0;
                int e2 = -1, e3 = -1;
                for (int k = 0; k < kP; ++k)
                    if (k != e && head[k] == head[e]) e2 = k;  // the other edge into head(e)
                if (e2 < 0 || side[e2] >= 0) break;
                side[e2] = 1;
                for (int k = 0; k < kP; ++k)
                    if (k != e2 && tail[k] == tail[e2]) e3 = k;  // the other edge out of tail(e2)
                if (e3 < 0) break;
                e = e3;
            }
        }
        int n[2] = {0, 0};
        for (int k = 0; k < kP; ++k) {
            if (side[k] < 0 || n[side[k]] >= kP / 2) return set_error(DMRG_E_STATE, "pair schedule: unbalanced split");
            const int slot = side[k] * (kP / 2) + n[side[k]]++;
            const int seated_first = seat_column(k, r);  // the column in seat k (seat lane k)
            tab[r * kP + slot] = (uint32_t)(pa[k] | pb[k] << 6 | (first[k] != pa[k] ? 1 : 0) << 12 | k << 13 |
                                            (seated_first != first[k] ? 1 : 0) << 18);
        }
        for (int h = 0; h < 2; ++h) {
            unsigned fm = 0, sm = 0;
            for (int l = 0; l < kP / 2; ++l) {
                const unsigned e = tab[r * kP + h * (kP / 2) + l];
                const int a = e & 63, b = (e >> 6) & 63, f = (e >> 12) & 1;
                fm |= 1u << ((f ? b : a) % kR);
                sm |= 1u << ((f ? a : b) % kR);
                ++met[a * kPair + b];
            }
            if (fm != 0xFFFFu || sm != 0xFFFFu) return set_error(DMRG_E_STATE, "pair schedule: bank collision");
        }
    }
    for (int a = 0; a < kPair; ++a)
        for (int b = a + 1; b < kPair; ++b)
            if (met[a * kPair + b] != 1) return set_error(DMRG_E_STATE, "pair schedule: pair (%d, %d) missed", a, b);
    return DMRG_OK;
}

const std::vector<uint32_t>* pair_schedule() {
    static std::vector<uint32_t> tab;
    static const int rc = build_pair_schedule(tab);
    return rc == DMRG_OK ? &tab : nullptr;
}

}  // namespace

int BatchedSvd::plan(const std::vector<int>& m, const std::vector<int>& n, cudaStream_t st) {
    probs.clear();
    tiles.clear();
    tile_first.clear();
    index.assign(m.size(), -1);
    int64_t woff = 0, qoff = 0, soff = 0;
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
        tile_first.push_back((int)tiles.size());
        for (int bi = 0; bi < nb; ++bi)
            for (int bj = bi; bj < nb; ++bj) tiles.push_back(SvdTile{(int)probs.size(), bi, bj, 0});
        probs.push_back(p);
    }
    tile_first.push_back((int)tiles.size());
    // Capacities.  A sweep holds at most every block pair of a problem plus one
    // pair per block for blocks unconverged only within themselves; a round at
    // most nbe / 2 pairs per problem.  Row ranges of the Gram items: at least
    // kGramMinRows rows each, fewer items than ~4 per SM in the widest round
    // (bounds the partial-Gram buffer).
    int64_t widest = 0, sweep_tasks = 0, sweep_gram = 0, sweep_rot = 0, round_tasks = 0;
    for (const SvdProblem& p : probs) {
        widest += (int64_t)p.rows * (p.nbe / 2);
        round_tasks += p.nbe / 2;
    }
    gram_rows = (int)std::max<int64_t>(kGramMinRows, ((widest / 600 + 31) / 32) * 32);
    int64_t round_gram = 0;
    for (const SvdProblem& p : probs) {
        const int64_t pairs = (int64_t)p.nbe * (p.nbe - 1) / 2 + p.nbe;
        const int64_t gi = (p.rows + gram_rows - 1) / gram_rows;
        const int64_t ri = (p.rows + kPair - 1) / kPair + (p.cols + kPair - 1) / kPair;
        sweep_tasks += pairs;
        sweep_gram += pairs * gi;
        sweep_rot += pairs * ri;
        round_gram += (int64_t)(p.nbe / 2) * gi;
    }
    max_tasks = (int)sweep_tasks;
    max_gram = (int)sweep_gram;
    max_rot = (int)sweep_rot;
    max_round_tasks = (int)round_tasks;
    max_round_gram = (int)round_gram;
    DMRG_TRY(d_w.alloc((size_t)std::max<int64_t>(woff, 1) * sizeof(double)));
    DMRG_TRY(d_q.alloc((size_t)std::max<int64_t>(qoff, 1) * sizeof(double)));
    DMRG_TRY(d_s.alloc((size_t)std::max<int64_t>(2 * soff, 1) * sizeof(double)));
    DMRG_TRY(d_perm.alloc((size_t)std::max<int64_t>(soff, 1) * sizeof(int)));
    DMRG_TRY(d_fro2.alloc(std::max<size_t>(probs.size(), 1) * sizeof(double)));
    DMRG_TRY(d_expo.alloc(std::max<size_t>(probs.size(), 1) * sizeof(int)));
    DMRG_TRY(d_part.alloc(std::max<size_t>(probs.size(), 1) * 2 * kSlices * sizeof(double)));
    DMRG_TRY(d_sign.alloc((size_t)std::max<int64_t>(soff, 1) * sizeof(double)));
    DMRG_TRY(d_colmap.alloc((size_t)std::max<int64_t>(soff, 1) * sizeof(int)));
    DMRG_TRY(d_norm.alloc((size_t)std::max<int64_t>(soff, 1) * sizeof(double)));
    DMRG_TRY(d_bm.alloc(std::max<size_t>(tiles.size(), 1) * sizeof(double)));
    if (!d_sched.ptr) {
        const std::vector<uint32_t>* sched = pair_schedule();
        if (!sched) return set_error(DMRG_E_STATE, "no pair schedule");
        DMRG_TRY(upload(d_sched, *sched, st));
    }
    DMRG_TRY(upload(d_probs, probs, st));
    DMRG_TRY(upload(d_tiles, tiles, st));
    DMRG_TRY(d_tasks.alloc(std::max<size_t>(max_tasks, 1) * sizeof(SvdTask)));
    DMRG_TRY(d_gram_items.alloc(std::max<size_t>(max_gram, 1) * sizeof(SvdItem)));
    DMRG_TRY(d_rot_items.alloc(std::max<size_t>(max_rot, 1) * sizeof(SvdItem)));
    DMRG_TRY(d_gpart.alloc((size_t)std::max(max_round_gram, 1) * kPair * kPair * sizeof(double)));
    DMRG_TRY(d_rot.alloc((size_t)std::max(max_round_tasks, 1) * kPair * kPair * sizeof(double)));
    DMRG_TRY(d_skip.alloc((size_t)std::max(max_round_tasks, 1) * sizeof(int)));
    DMRG_CUDA_TRY(cudaFuncSetAttribute(solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(SvdSmem)));
    static_assert(sizeof(SvdSmem) <= 227 * 1024, "pair solve shared memory");
    DMRG_CUDA_TRY(cudaFuncSetAttribute(rotate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRotSmem));
    return DMRG_OK;
}

void BatchedSvd::add_task(int problem, int bi, int bj) {
    const SvdProblem& p = probs[problem];
    const int t = (int)tasks.size();
    SvdTask task{problem, bi, bj, (int)gram_items.size() - round_gram_first.back(), 0};
    for (int r0 = 0; r0 < p.rows; r0 += gram_rows)
        gram_items.push_back(SvdItem{t, 0, r0, std::min(p.rows, r0 + gram_rows)});
    task.g_count = (int)gram_items.size() - round_gram_first.back() - task.g_first;
    tasks.push_back(task);
    for (int r0 = 0; r0 < p.rows; r0 += kPair) rot_items.push_back(SvdItem{t, 0, r0, std::min(p.rows, r0 + kPair)});
    for (int r0 = 0; r0 < p.cols; r0 += kPair) rot_items.push_back(SvdItem{t, 1, r0, std::min(p.cols, r0 + kPair)});
}

// Rounds of one problem's sweep: its unconverged block pairs (measure > tol) as
// a sequence of matchings, and every block unconverged within itself in some
// pair.  Two candidates, the fewer rounds kept: the round-robin order over nbe
// blocks restricted to those pairs, and a greedy matching by decreasing measure.
static std::vector<std::vector<std::pair<int, int>>> problem_rounds(const SvdProblem& p, const double* bm,
                                                                     double tol) {
    const int nb = (p.cols + kBlk - 1) / kBlk;
    auto at = [&](int i, int j) {  // tiles of a problem: bi <= bj, row-major over bi
        if (i > j) std::swap(i, j);
        return bm[i * nb - i * (i - 1) / 2 + (j - i)];
    };
    std::vector<std::pair<double, std::pair<int, int>>> cross;
    std::vector<int> internal;
    for (int i = 0; i < nb; ++i) {
        if (at(i, i) > tol) internal.push_back(i);
        for (int j = i + 1; j < nb; ++j)
            if (at(i, j) > tol) cross.push_back({at(i, j), {i, j}});
    }
    using Rounds = std::vector<std::vector<std::pair<int, int>>>;
    auto cover = [&](Rounds& rounds) {  // every internally unconverged block in some pair
        std::vector<char> seen(p.nbe, 0);
        for (const auto& rd : rounds)
            for (const auto& pr : rd) seen[pr.first] = seen[pr.second] = 1;
        for (int i : internal) {
            if (seen[i]) continue;
            bool placed = false;
            for (auto& rd : rounds) {
                std::vector<char> used(p.nbe, 0);
                for (const auto& pr : rd) used[pr.first] = used[pr.second] = 1;
                if (used[i]) continue;
                for (int j = 0; j < p.nbe && !placed; ++j)
                    if (j != i && !used[j]) {
                        rd.push_back({std::min(i, j), std::max(i, j)});
                        seen[j] = 1;
                        placed = true;
                    }
                if (placed) break;
            }
            if (!placed) {
                const int j = (i + 1) % p.nbe;
                rounds.push_back({{std::min(i, j), std::max(i, j)}});
                seen[j] = 1;
            }
            seen[i] = 1;
        }
    };
    Rounds rr;
    {
        std::vector<char> need((size_t)p.nbe * p.nbe, 0);
        for (const auto& c : cross) need[c.second.first * p.nbe + c.second.second] = 1;
        for (int r = 0; r < p.nbe - 1; ++r) {
            std::vector<std::pair<int, int>> rd;
            for (int k = 0; k < p.nbe / 2; ++k) {
                int i, j;
                rr_pair(r, k, p.nbe, i, j);
                if (need[i * p.nbe + j]) rd.push_back({i, j});
            }
            if (!rd.empty()) rr.push_back(rd);
        }
        cover(rr);
    }
    Rounds gr;
    {
        std::sort(cross.begin(), cross.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
        std::vector<std::vector<char>> used;
        for (const auto& c : cross) {
            const int i = c.second.first, j = c.second.second;
            size_t r = 0;
            for (; r < gr.size(); ++r)
                if (!used[r][i] && !used[r][j]) break;
            if (r == gr.size()) {
                gr.emplace_back();
                used.emplace_back(p.nbe, 0);
            }
            gr[r].push_back({i, j});
            used[r][i] = used[r][j] = 1;
        }
        cover(gr);
    }
    return gr.size() < rr.size() ? gr : rr;
}

int BatchedSvd::schedule(const std::vector<double>& bm) {
    tasks.clear();
    gram_items.clear();
    rot_items.clear();
    round_first.clear();
    round_gram_first.clear();
    round_rot_first.clear();
    std::vector<std::vector<std::vector<std::pair<int, int>>>> per(probs.size());
    size_t rounds = 0;
    for (size_t pi = 0; pi < probs.size(); ++pi) {
        const double tol = 2.0 * DBL_EPSILON * std::sqrt((double)probs[pi].rows);
        per[pi] = problem_rounds(probs[pi], bm.data() + tile_first[pi], tol);
        rounds = std::max(rounds, per[pi].size());
    }
    for (size_t r = 0; r < rounds; ++r) {
        round_first.push_back((int)tasks.size());
        round_gram_first.push_back((int)gram_items.size());
        round_rot_first.push_back((int)rot_items.size());
        for (size_t pi = 0; pi < probs.size(); ++pi)
            if (r < per[pi].size())
                for (const auto& pr : per[pi][r]) add_task((int)pi, pr.first, pr.second);
    }
    round_first.push_back((int)tasks.size());
    round_gram_first.push_back((int)gram_items.size());
    round_rot_first.push_back((int)rot_items.size());
    return (int)rounds;
}

// Appends, for each problem whose last measure was above tol: m, n, rows,
// cols, transposed (int32), fro2 and the measure (float64), then its input and
// final working matrices (rows x cols float64, column-major).
void BatchedSvd::dump_unconverged(const char* path, const DeviceBuffer& w_in, const std::vector<double>& worst,
                                  cudaStream_t st) {
    std::FILE* f = std::fopen(path, "ab");
    if (!f) return;
    std::vector<double> fro2(probs.size());
    cudaMemcpyAsync(fro2.data(), d_fro2.ptr, fro2.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    for (size_t i = 0; i < probs.size(); ++i) {
        const SvdProblem& p = probs[i];
        if (worst[i] <= 2.0 * DBL_EPSILON * std::sqrt((double)p.rows)) continue;
        const size_t cnt = (size_t)p.rows * p.cols;
        std::vector<double> a(cnt), b(cnt);
        cudaMemcpyAsync(a.data(), w_in.as<double>() + p.w_off, cnt * sizeof(double), cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(b.data(), d_w.as<double>() + p.w_off, cnt * sizeof(double), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        const int hdr[5] = {p.m, p.n, p.rows, p.cols, p.transposed};
        const double val[2] = {fro2[i], worst[i]};
        std::fwrite(hdr, sizeof(int), 5, f);
        std::fwrite(val, sizeof(double), 2, f);
        std::fwrite(a.data(), sizeof(double), cnt, f);
        std::fwrite(b.data(), sizeof(double), cnt, f);
    }
    std::fclose(f);
}

int BatchedSvd::run(cudaStream_t st, int* sweeps_out) {
    if (probs.empty()) {
        if (sweeps_out) *sweeps_out = 0;
        return DMRG_OK;
    }
    const int np = (int)probs.size();
    // DMRG_SVD_FAIL_DUMP=path: keep the input, and if the sweeps do not converge
    // write every unconverged sector's input and final working matrix to path
    // (diagnostics only; see dump_unconverged)
    static const char* fail_dump = std::getenv("DMRG_SVD_FAIL_DUMP");
    DeviceBuffer w_in;
    if (fail_dump) {
        DMRG_TRY(w_in.alloc(d_w.bytes));
        DMRG_CUDA_TRY(cudaMemcpyAsync(w_in.ptr, d_w.ptr, d_w.bytes, cudaMemcpyDeviceToDevice, st));
    }
    const dim3 sliced(np, kSlices);
    DMRG_LAUNCH init_identity_kernel<<<sliced, 256, 0, st>>>(d_probs.as<SvdProblem>(), d_q.as<double>());
    DMRG_LAUNCH slice_max_kernel<<<sliced, 256, 0, st>>>(d_probs.as<SvdProblem>(), d_w.as<double>(), d_part.as<double>());
    DMRG_LAUNCH prescale_kernel<<<sliced, 256, 0, st>>>(d_probs.as<SvdProblem>(), d_w.as<double>(), d_part.as<double>(),
                                                        d_expo.as<int>(), d_part.as<double>() + (int64_t)np * kSlices);
    DMRG_LAUNCH fro2_kernel<<<(np + 127) / 128, 128, 0, st>>>(d_part.as<double>() + (int64_t)np * kSlices, np,
                                                              d_fro2.as<double>());
    static const bool debug = std::getenv("DMRG_SVD_DEBUG") != nullptr;  // per-sweep convergence to stderr
    int max_cols = 0;
    for (const SvdProblem& p : probs) max_cols = std::max(max_cols, p.cols);
    const dim3 colgrid(np, (max_cols + 7) / 8);
    const dim3 rankgrid(np, (max_cols + 255) / 256);
    std::vector<double> bm(tiles.size()), worst(np);
    const int max_sweeps = g_max_sweeps.load();
    auto t_sweep = std::chrono::steady_clock::now();
    int sweep = 0;
    bool converged = false;
    for (;; ++sweep) {
        // the sweep visits columns in descending norm order: blocks hold columns of
        // similar size, which keeps the many tiny singular values of a noise-expanded
        // tensor from converging only linearly; then every block pair is measured
        DMRG_LAUNCH colnorm_kernel<<<colgrid, 256, 0, st>>>(d_probs.as<SvdProblem>(), d_w.as<double>(), d_norm.as<double>());
        DMRG_LAUNCH rank_kernel<<<rankgrid, 256, 0, st>>>(d_probs.as<SvdProblem>(), d_norm.as<double>(), d_colmap.as<int>(),
                                                    nullptr);
        DMRG_LAUNCH measure_kernel<<<(int)tiles.size(), 128, 0, st>>>(
            d_probs.as<SvdProblem>(), d_tiles.as<SvdTile>(), d_colmap.as<int>(), d_w.as<double>(),
            d_norm.as<double>(), d_fro2.as<double>(), d_bm.as<double>());
        DMRG_CUDA_TRY(cudaGetLastError());
        DMRG_CUDA_TRY(cudaMemcpyAsync(bm.data(), d_bm.ptr, bm.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        DMRG_CUDA_TRY(cudaStreamSynchronize(st));
        for (int i = 0; i < np; ++i) {
            worst[i] = 0.0;
            for (int k = tile_first[i]; k < tile_first[i + 1]; ++k) worst[i] = std::max(worst[i], bm[k]);
        }
        const int rounds = schedule(bm);
        if (debug) {
            int wi = 0;
            for (int i = 1; i < np; ++i)
                if (worst[i] > worst[wi]) wi = i;
            const auto now = std::chrono::steady_clock::now();
            std::fprintf(stderr, "svd sweep %d: %.2f ms, worst %.3e (sector %d x %d), %d rounds\n", sweep,
                         std::chrono::duration<double, std::milli>(now - t_sweep).count(), worst[wi], probs[wi].m,
                         probs[wi].n, rounds);
            t_sweep = now;
        }
        if (rounds == 0) {
            converged = true;
            break;
        }
        if (sweep >= max_sweeps) break;
        int widest_round = 0, widest_gram = 0;
        for (int r = 0; r < rounds; ++r) {
            widest_round = std::max(widest_round, round_first[r + 1] - round_first[r]);
            widest_gram = std::max(widest_gram, round_gram_first[r + 1] - round_gram_first[r]);
        }
        if ((int)tasks.size() > max_tasks || (int)gram_items.size() > max_gram || (int)rot_items.size() > max_rot ||
            widest_round > max_round_tasks || widest_gram > max_round_gram)
            return set_error(DMRG_E_STATE, "Jacobi SVD schedule exceeds its plan");
        DMRG_CUDA_TRY(cudaMemcpyAsync(d_tasks.ptr, tasks.data(), tasks.size() * sizeof(SvdTask), cudaMemcpyHostToDevice, st));
        DMRG_CUDA_TRY(cudaMemcpyAsync(d_gram_items.ptr, gram_items.data(), gram_items.size() * sizeof(SvdItem),
                                      cudaMemcpyHostToDevice, st));
        DMRG_CUDA_TRY(cudaMemcpyAsync(d_rot_items.ptr, rot_items.data(), rot_items.size() * sizeof(SvdItem),
                                      cudaMemcpyHostToDevice, st));
        for (int r = 0; r < rounds; ++r) {
            const int nt = round_first[r + 1] - round_first[r];
            const int ng = round_gram_first[r + 1] - round_gram_first[r];
            const int nr = round_rot_first[r + 1] - round_rot_first[r];
            if (nt == 0) continue;
            DMRG_LAUNCH gram_kernel<<<ng, 128, 0, st>>>(d_probs.as<SvdProblem>(), d_tasks.as<SvdTask>(),
                                                        d_gram_items.as<SvdItem>() + round_gram_first[r],
                                                        d_colmap.as<int>(), d_w.as<double>(), d_gpart.as<double>());
            DMRG_LAUNCH solve_kernel<<<nt, kThreads, sizeof(SvdSmem), st>>>(
                d_probs.as<SvdProblem>(), d_tasks.as<SvdTask>(), round_first[r], d_gpart.as<double>(),
                d_fro2.as<double>(), d_rot.as<double>(), d_skip.as<int>(), d_sched.as<uint32_t>(), kInnerSweeps);
            DMRG_LAUNCH rotate_kernel<<<nr, 128, kRotSmem, st>>>(d_probs.as<SvdProblem>(), d_tasks.as<SvdTask>(),
                                                                 d_rot_items.as<SvdItem>() + round_rot_first[r],
                                                                 round_first[r], d_rot.as<double>(), d_skip.as<int>(),
                                                                 d_colmap.as<int>(), d_w.as<double>(), d_q.as<double>());
        }
        DMRG_CUDA_TRY(cudaGetLastError());
    }
    if (!converged) {
        if (fail_dump) dump_unconverged(fail_dump, w_in, worst, st);
        int wi = 0;
        for (int i = 1; i < np; ++i)
            if (worst[i] > worst[wi]) wi = i;
        return set_error(DMRG_E_NUMERIC, "Jacobi SVD did not converge in %d sweeps (sector %d x %d: off-diagonal %.3e)",
                         max_sweeps, probs[wi].m, probs[wi].n, worst[wi]);
    }
    // singular values = final column norms, sorted
    DMRG_LAUNCH colnorm_kernel<<<colgrid, 256, 0, st>>>(d_probs.as<SvdProblem>(), d_w.as<double>(), d_norm.as<double>());
    DMRG_LAUNCH rank_kernel<<<rankgrid, 256, 0, st>>>(d_probs.as<SvdProblem>(), d_norm.as<double>(), d_perm.as<int>(), d_s.as<double>());
    DMRG_LAUNCH sign_kernel<<<colgrid, 256, 0, st>>>(d_probs.as<SvdProblem>(), d_w.as<double>(),
                                                               d_q.as<double>(), d_perm.as<int>(), d_sign.as<double>());
    DMRG_LAUNCH unscale_kernel<<<dim3(np, 32), 256, 0, st>>>(d_probs.as<SvdProblem>(), d_expo.as<int>(),
                                                             d_w.as<double>(), d_s.as<double>());
    DMRG_CUDA_TRY(cudaGetLastError());
    if (sweeps_out) *sweeps_out = sweep;  // sweeps that rotated
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

extern "C" int dmrg_svd_set_max_sweeps(int sweeps) {
    dmrg::g_max_sweeps.store(sweeps > 0 ? sweeps : dmrg::kMaxSweeps);
    return DMRG_OK;
}

extern "C" int dmrg_svd_plan_rounds(int cols, const double* bm, double tol, int cap, int* pairs, int* n_pairs,
                                    int* n_rounds) {
    if (cols <= 0 || !bm || !n_pairs || !n_rounds || (cap > 0 && !pairs))
        return dmrg::set_error(DMRG_E_ARG, "invalid argument");
    dmrg::SvdProblem p{};
    p.rows = p.cols = p.m = p.n = cols;
    const int nb = (cols + dmrg::kBlk - 1) / dmrg::kBlk;
    p.nbe = std::max(2, nb + (nb & 1));
    const auto rounds = dmrg::problem_rounds(p, bm, tol);
    int k = 0;
    for (size_t r = 0; r < rounds.size(); ++r)
        for (const auto& pr : rounds[r]) {
            if (k < cap) pairs[k] = (int)r << 16 | pr.first << 8 | pr.second;
            ++k;
        }
    *n_pairs = k;
    *n_rounds = (int)rounds.size();
    return k <= cap ? DMRG_OK : dmrg::set_error(DMRG_E_ARG, "%d pairs, room for %d", k, cap);
}

extern "C" int dmrg_svd_pair_schedule(unsigned int* out) {
    if (!out) return dmrg::set_error(DMRG_E_ARG, "null argument");
    const std::vector<uint32_t>* tab = dmrg::pair_schedule();
    if (!tab) return DMRG_E_STATE;
    std::memcpy(out, tab->data(), tab->size() * sizeof(uint32_t));
    return DMRG_OK;
}
