// FP64 grouped multi-term block GEMM on the FP64 tensor path (DMMA,
// mma.sync.m8n8k4.f64).  tcgen05 has no f64 kind, so this is the sm_100a FP64
// contraction engine.
//
// CTA: 128 threads (2x2 warps), 64x64 output tile, k-step 16, two shared-memory
// stages filled by 8-byte cp.async (block leading dimensions are arbitrary, so
// neither 16-byte vector loads nor TMA tensor maps apply to the raw blocks).
// Each warp owns a 32x32 sub-tile = 4x4 DMMA tiles, 32 FP64 accumulators per
// thread.  Shared tiles are stored in the operand's global orientation with a
// 4-double row pad, which makes every fragment read conflict-free.
#include <algorithm>
#include <numeric>

#include "gemm.cuh"

namespace dmrg {
namespace {

constexpr int BM = 64, BK = 16, NT = 128;  // tile N is also 64 (2 warps x 32)
constexpr int SA = BK + 4;            // stride of a [64][16] tile
constexpr int SB = BM + 4;            // stride of a [16][64] tile
constexpr int STAGE = BM * SA;        // 1280 >= BK * SB = 1088

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool valid) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int src_size = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_size)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <bool TA, bool TB>
__device__ __forceinline__ void load_stage(double* As, double* Bs, const double* __restrict__ A,
                                           const double* __restrict__ B, const GemmTerm& t, int k0,
                                           int m0, int n0, int m, int n, int tid) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int idx = tid + NT * i;
        const int r = TA ? (idx & 63) : (idx >> 4);
        const int c = TA ? (idx >> 6) : (idx & 15);
        const bool v = (m0 + r < m) && (k0 + c < t.k);
        const int64_t off = TA ? (int64_t)(k0 + c) * t.lda + (m0 + r) : (int64_t)(m0 + r) * t.lda + (k0 + c);
        cp_async8(TA ? (As + c * SB + r) : (As + r * SA + c), v ? (A + t.a_off + off) : A, v);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int idx = tid + NT * i;
        const int nn = TB ? (idx >> 4) : (idx & 63);
        const int c = TB ? (idx & 15) : (idx >> 6);
        const bool v = (n0 + nn < n) && (k0 + c < t.k);
        const int64_t off = TB ? (int64_t)(n0 + nn) * t.ldb + (k0 + c) : (int64_t)(k0 + c) * t.ldb + (n0 + nn);
        cp_async8(TB ? (Bs + nn * SA + c) : (Bs + c * SB + nn), v ? (B + t.b_off + off) : B, v);
    }
}

template <bool TA, bool TB>
__device__ __forceinline__ void compute_stage(const double* As, const double* Bs, double (&acc)[4][4][2],
                                              double scale, int wm, int wn, int lane) {
    const int fr = lane >> 2, fc = lane & 3;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int row = wm * 32 + i * 8 + fr, col = kk + fc;
            a[i] = (TA ? As[col * SB + row] : As[row * SA + col]) * scale;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int kr = kk + fc, nc = wn * 32 + j * 8 + fr;
            b[j] = TB ? Bs[nc * SA + kr] : Bs[kr * SB + nc];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(NT) gemm_f64_kernel(const double* __restrict__ A, const double* __restrict__ B,
                                                      double* __restrict__ C, double* __restrict__ Caux,
                                                      const GemmTerm* __restrict__ terms,
                                                      const GemmGroup* __restrict__ groups,
                                                      const GemmTile* __restrict__ tiles, int accumulate) {
    __shared__ __align__(16) double smA[2][STAGE];
    __shared__ __align__(16) double smB[2][STAGE];
    const GemmTile tile = tiles[blockIdx.x];
    const GemmGroup g = groups[tile.group];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp >> 1, wn = warp & 1;

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    int t = g.t0;
    if (t < g.t1) {
        GemmTerm cur = terms[t];
        int k0 = 0, stage = 0;
        double sc_cur = cur.scale;
        load_stage<TA, TB>(smA[0], smB[0], A, B, cur, 0, tile.m0, tile.n0, g.m, g.n, tid);
        cp_async_commit();
        for (;;) {
            int nk0 = k0 + BK, nt = t;
            GemmTerm nxt = cur;
            if (nk0 >= cur.k) {
                nt = t + 1;
                nk0 = 0;
                if (nt < g.t1) nxt = terms[nt];
            }
            const bool has_next = nt < g.t1;
            double sc_nxt = nxt.scale;
            if (has_next) {
                load_stage<TA, TB>(smA[stage ^ 1], smB[stage ^ 1], A, B, nxt, nk0, tile.m0, tile.n0, g.m, g.n,
                                   tid);
                cp_async_commit();
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            compute_stage<TA, TB>(smA[stage], smB[stage], acc, sc_cur, wm, wn, lane);
            __syncthreads();
            if (!has_next) break;
            stage ^= 1;
            t = nt;
            k0 = nk0;
            cur = nxt;
            sc_cur = sc_nxt;
        }
    }

    const int fr = lane >> 2, fc = lane & 3;
    const bool acc_out = accumulate && g.cbuf == 0;
    double* Cb = g.cbuf ? Caux : C;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int row = tile.m0 + wm * 32 + i * 8 + fr;
        if (row >= g.m) continue;
        double* crow = Cb + g.c_off + (int64_t)row * g.ldc;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int col = tile.n0 + wn * 32 + j * 8 + fc * 2 + e;
                if (col < g.n) crow[col] = acc_out ? crow[col] + acc[i][j][e] : acc[i][j][e];
            }
        }
    }
}

// Grid (element slices, split groups): C[c_off + r*ldc + c] (+)= sum over the
// group's chunks, in chunk order (deterministic).
__global__ void __launch_bounds__(256) split_reduce_kernel(double* __restrict__ C, const double* __restrict__ Caux,
                                                           const GemmSplit* __restrict__ splits, int accumulate) {
    const GemmSplit s = splits[blockIdx.y];
    const int64_t tile = (int64_t)s.m * s.n;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tile; e += (int64_t)gridDim.x * blockDim.x) {
        double v = 0.0;
        for (int c = 0; c < s.chunks; ++c) v += Caux[s.aux_off + c * tile + e];
        const int r = (int)(e / s.n), col = (int)(e % s.n);
        double* p = C + s.c_off + (int64_t)r * s.ldc + col;
        *p = accumulate ? *p + v : v;
    }
}

}  // namespace

int GemmSchedule::check_bounds(int64_t a_size, int64_t b_size, int64_t c_size) const {
    for (const GemmGroup& g : groups) {
        if (g.m <= 0 || g.n <= 0) continue;
        if (g.c_off < 0 || g.c_off + (int64_t)(g.m - 1) * g.ldc + g.n > c_size || g.n > g.ldc)
            return set_error(DMRG_E_ARG, "GEMM output %lld (%dx%d, ld %d) outside %lld", (long long)g.c_off, g.m, g.n,
                             g.ldc, (long long)c_size);
        for (int ti = g.t0; ti < g.t1; ++ti) {
            const GemmTerm& t = terms[ti];
            if (t.k <= 0) continue;
            const int64_t ae = ta ? t.a_off + (int64_t)(t.k - 1) * t.lda + g.m : t.a_off + (int64_t)(g.m - 1) * t.lda + t.k;
            const int64_t be = tb ? t.b_off + (int64_t)(g.n - 1) * t.ldb + t.k : t.b_off + (int64_t)(t.k - 1) * t.ldb + g.n;
            if (t.a_off < 0 || ae > a_size || t.b_off < 0 || be > b_size)
                return set_error(DMRG_E_ARG, "GEMM operand outside its buffer (A end %lld of %lld, B end %lld of %lld)",
                                 (long long)ae, (long long)a_size, (long long)be, (long long)b_size);
        }
    }
    return DMRG_OK;
}

int GemmSchedule::finalize(int tile_m, int tile_n, int tile_k, cudaStream_t stream, int num_sms) {
    tiles.clear();
    exec_groups.clear();
    splits.clear();
    aux_size = 0;
    this->tile_m = tile_m;
    this->tile_n = tile_n;
    this->tile_k = tile_k;
    auto ksteps_of = [&](int t) { return (terms[t].k + tile_k - 1) / tile_k; };
    auto ntiles_of = [&](const GemmGroup& g) {
        return (int64_t)((g.m + tile_m - 1) / tile_m) * ((g.n + tile_n - 1) / tile_n);
    };
    // balanced share of k-steps per CTA (4 resident CTAs per SM, two waves)
    int64_t total = 0;
    for (const GemmGroup& g : groups) {
        if (g.m <= 0 || g.n <= 0) continue;
        int64_t ks = 0;
        for (int t = g.t0; t < g.t1; ++t) ks += ksteps_of(t);
        total += ks * ntiles_of(g);
    }
    const int64_t share = num_sms > 0 ? std::max<int64_t>(16, total / ((int64_t)num_sms * 8)) : 0;
    for (const GemmGroup& g : groups) {
        if (g.m <= 0 || g.n <= 0 || g.t1 <= g.t0) continue;
        int64_t ks = 0;
        for (int t = g.t0; t < g.t1; ++t) ks += ksteps_of(t);
        if (share == 0 || ks <= 2 * share || g.t1 - g.t0 < 2) {
            exec_groups.push_back(g);
            continue;
        }
        // split the term range into contiguous chunks of about `share` k-steps
        GemmSplit sp{g.c_off, aux_size, g.ldc, g.m, g.n, 0};
        int t0 = g.t0;
        int64_t acc = 0;
        for (int t = g.t0; t < g.t1; ++t) {
            acc += ksteps_of(t);
            if (acc >= share || t + 1 == g.t1) {
                GemmGroup c{aux_size + (int64_t)sp.chunks * g.m * g.n, g.n, g.m, g.n, t0, t + 1, 1};
                exec_groups.push_back(c);
                sp.chunks++;
                t0 = t + 1;
                acc = 0;
            }
        }
        aux_size += (int64_t)sp.chunks * g.m * g.n;
        splits.push_back(sp);
    }
    for (int gi = 0; gi < (int)exec_groups.size(); ++gi) {
        const GemmGroup& g = exec_groups[gi];
        int ks = 0;
        for (int t = g.t0; t < g.t1; ++t) ks += ksteps_of(t);
        for (int m0 = 0; m0 < g.m; m0 += tile_m)
            for (int n0 = 0; n0 < g.n; n0 += tile_n) tiles.push_back(GemmTile{gi, m0, n0, ks});
    }
    std::stable_sort(tiles.begin(), tiles.end(), [](const GemmTile& a, const GemmTile& b) { return a.cost > b.cost; });
    DMRG_TRY(upload(d_terms, terms, stream));
    DMRG_TRY(upload(d_groups, exec_groups, stream));
    DMRG_TRY(upload(d_tiles, tiles, stream));
    DMRG_TRY(upload(d_splits, splits, stream));
    DMRG_TRY(aux.alloc((size_t)std::max<int64_t>(aux_size, 1) * sizeof(double)));
    return DMRG_OK;
}

int launch_gemm_f64(const GemmSchedule& s, const double* A, const double* B, double* C, bool accumulate,
                    cudaStream_t stream) {
    if (s.tiles.empty()) return DMRG_OK;
    const int n = (int)s.tiles.size();
    const auto* tr = s.d_terms.as<GemmTerm>();
    const auto* gr = s.d_groups.as<GemmGroup>();
    const auto* tl = s.d_tiles.as<GemmTile>();
    const int acc = accumulate ? 1 : 0;
    double* X = s.aux.as<double>();
    if (!s.ta && !s.tb) DMRG_LAUNCH gemm_f64_kernel<false, false><<<n, NT, 0, stream>>>(A, B, C, X, tr, gr, tl, acc);
    else if (s.ta && !s.tb) DMRG_LAUNCH gemm_f64_kernel<true, false><<<n, NT, 0, stream>>>(A, B, C, X, tr, gr, tl, acc);
    else if (!s.ta && s.tb) DMRG_LAUNCH gemm_f64_kernel<false, true><<<n, NT, 0, stream>>>(A, B, C, X, tr, gr, tl, acc);
    else DMRG_LAUNCH gemm_f64_kernel<true, true><<<n, NT, 0, stream>>>(A, B, C, X, tr, gr, tl, acc);
    if (!s.splits.empty()) {
        int64_t biggest = 0;
        for (const GemmSplit& sp : s.splits) biggest = std::max<int64_t>(biggest, (int64_t)sp.m * sp.n);
        const int gx = (int)std::min<int64_t>((biggest + 255) / 256, 64);
        DMRG_LAUNCH split_reduce_kernel<<<dim3(gx, (unsigned)s.splits.size()), 256, 0, stream>>>(C, X, s.d_splits.as<GemmSplit>(),
                                                                                     acc);
    }
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int launch_gemm_f64_tables(const GemmTerm* terms, const GemmGroup* groups, const GemmTile* tiles, int ntiles,
                           bool ta, bool tb, const double* A, const double* B, double* C, bool accumulate,
                           cudaStream_t stream) {
    // Same kernel as launch_gemm_f64, with device tables supplied by the caller
    // (no split-K groups: every group writes C directly).
    if (ntiles <= 0) return DMRG_OK;
    const int acc = accumulate ? 1 : 0;
    if (!ta && !tb) DMRG_LAUNCH gemm_f64_kernel<false, false><<<ntiles, NT, 0, stream>>>(A, B, C, nullptr, terms, groups, tiles, acc);
    else if (ta && !tb) DMRG_LAUNCH gemm_f64_kernel<true, false><<<ntiles, NT, 0, stream>>>(A, B, C, nullptr, terms, groups, tiles, acc);
    else if (!ta && tb) DMRG_LAUNCH gemm_f64_kernel<false, true><<<ntiles, NT, 0, stream>>>(A, B, C, nullptr, terms, groups, tiles, acc);
    else DMRG_LAUNCH gemm_f64_kernel<true, true><<<ntiles, NT, 0, stream>>>(A, B, C, nullptr, terms, groups, tiles, acc);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

}  // namespace dmrg
