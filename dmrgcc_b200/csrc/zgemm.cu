// Complex grouped block GEMM on the FP64 tensor path (see zgemm.cuh).
//
// A complex product is four real DMMA products (mma.sync.m8n8k4.f64):
//   C_re += A_re B_re - A_im B_im,   C_im += A_re B_im + A_im B_re,
// with the term's complex scale folded into the A fragments and conjugation
// into the sign of the imaginary parts.  CTA: 128 threads (2 x 2 warps), a
// 64 x 32 complex output tile (each warp 32 x 16 = 4 x 2 DMMA tiles, a real and
// an imaginary accumulator pair per tile: 32 FP64 registers per thread), k-step
// 8, two shared-memory stages filled by 16-byte cp.async (one complex element
// each), zero-filled outside the block.
#include <algorithm>

#include "zgemm.cuh"

namespace dmrg {
namespace {

constexpr int ZM = 64, ZN = 32, ZK = 8, ZT = 128;
constexpr int APAD = ZK + 1;   // row stride (complex) of a [64][8] A tile
constexpr int ATPAD = ZM + 1;  // row stride of a [8][64] (transposed) A tile
constexpr int BPAD = ZN + 1;   // row stride of a [8][32] B tile
constexpr int BTPAD = ZK + 1;  // row stride of a [32][8] (transposed) B tile
constexpr int ASTAGE = ZM * APAD > ZK * ATPAD ? ZM * APAD : ZK * ATPAD;
constexpr int BSTAGE = ZK * BPAD > ZN * BTPAD ? ZK * BPAD : ZN * BTPAD;

__device__ __forceinline__ void cp_async16(double2* smem, const double2* gmem, bool valid) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int src_size = valid ? 16 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_size) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <bool TA, bool TB>
__device__ __forceinline__ void zload(double2* As, double2* Bs, const double2* __restrict__ A,
                                      const double2* __restrict__ B, const ZGemmTerm& t, int k0, int m0, int n0,
                                      int m, int n, int tid) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int idx = tid + ZT * i;
        const int r = TA ? (idx & 63) : (idx >> 3);
        const int c = TA ? (idx >> 6) : (idx & 7);
        const bool v = (m0 + r < m) && (k0 + c < t.k);
        const int64_t off = TA ? (int64_t)(k0 + c) * t.lda + (m0 + r) : (int64_t)(m0 + r) * t.lda + (k0 + c);
        cp_async16(TA ? (As + c * ATPAD + r) : (As + r * APAD + c), v ? (A + t.a_off + off) : A, v);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int idx = tid + ZT * i;
        const int nn = TB ? (idx >> 3) : (idx & 31);
        const int c = TB ? (idx & 7) : (idx >> 5);
        const bool v = (n0 + nn < n) && (k0 + c < t.k);
        const int64_t off = TB ? (int64_t)(n0 + nn) * t.ldb + (k0 + c) : (int64_t)(k0 + c) * t.ldb + (n0 + nn);
        cp_async16(TB ? (Bs + nn * BTPAD + c) : (Bs + c * BPAD + nn), v ? (B + t.b_off + off) : B, v);
    }
}

template <bool TA, bool TB>
__device__ __forceinline__ void zcompute(const double2* As, const double2* Bs, double (&re)[4][2][2],
                                         double (&im)[4][2][2], double s_re, double s_im, int conj, int wm, int wn,
                                         int lane) {
    const int fr = lane >> 2, fc = lane & 3;
    const double ca = (conj & 1) ? -1.0 : 1.0, cb = (conj & 2) ? -1.0 : 1.0;
#pragma unroll
    for (int kk = 0; kk < ZK; kk += 4) {
        double ar[4], ai[4], nai[4], br[2], bi[2];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int row = wm * 32 + i * 8 + fr, col = kk + fc;
            const double2 x = TA ? As[col * ATPAD + row] : As[row * APAD + col];
            const double xr = x.x, xi = ca * x.y;
            ar[i] = xr * s_re - xi * s_im;  // scale folded into A
            ai[i] = xr * s_im + xi * s_re;
            nai[i] = -ai[i];
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int kr = kk + fc, nc = wn * 16 + j * 8 + fr;
            const double2 y = TB ? Bs[nc * BTPAD + kr] : Bs[kr * BPAD + nc];
            br[j] = y.x;
            bi[j] = cb * y.y;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                dmma(re[i][j][0], re[i][j][1], ar[i], br[j]);
                dmma(re[i][j][0], re[i][j][1], nai[i], bi[j]);
                dmma(im[i][j][0], im[i][j][1], ar[i], bi[j]);
                dmma(im[i][j][0], im[i][j][1], ai[i], br[j]);
            }
    }
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(ZT) zgemm_kernel(const double2* __restrict__ A, const double2* __restrict__ B,
                                                   double2* __restrict__ C, const ZGemmTerm* __restrict__ terms,
                                                   const GemmGroup* __restrict__ groups,
                                                   const GemmTile* __restrict__ tiles, int accumulate) {
    __shared__ __align__(16) double2 smA[2][ASTAGE];
    __shared__ __align__(16) double2 smB[2][BSTAGE];
    const GemmTile tile = tiles[blockIdx.x];
    const GemmGroup g = groups[tile.group];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wm = warp >> 1, wn = warp & 1;
    double re[4][2][2], im[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) re[i][j][0] = re[i][j][1] = im[i][j][0] = im[i][j][1] = 0.0;

    int t = g.t0;
    if (t < g.t1) {
        ZGemmTerm cur = terms[t];
        int k0 = 0, stage = 0;
        zload<TA, TB>(smA[0], smB[0], A, B, cur, 0, tile.m0, tile.n0, g.m, g.n, tid);
        cp_commit();
        for (;;) {
            int nk0 = k0 + ZK, nt = t;
            ZGemmTerm nxt = cur;
            if (nk0 >= cur.k) {
                nt = t + 1;
                nk0 = 0;
                if (nt < g.t1) nxt = terms[nt];
            }
            const bool has_next = nt < g.t1;
            if (has_next) {
                zload<TA, TB>(smA[stage ^ 1], smB[stage ^ 1], A, B, nxt, nk0, tile.m0, tile.n0, g.m, g.n, tid);
                cp_commit();
                cp_wait<1>();
            } else {
                cp_wait<0>();
            }
            __syncthreads();
            zcompute<TA, TB>(smA[stage], smB[stage], re, im, cur.s_re, cur.s_im, cur.conj, wm, wn, lane);
            __syncthreads();
            if (!has_next) break;
            stage ^= 1;
            t = nt;
            k0 = nk0;
            cur = nxt;
        }
    }
    const int fr = lane >> 2, fc = lane & 3;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int row = tile.m0 + wm * 32 + i * 8 + fr;
        if (row >= g.m) continue;
        double2* crow = C + g.c_off + (int64_t)row * g.ldc;
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int col = tile.n0 + wn * 16 + j * 8 + fc * 2 + e;
                if (col >= g.n) continue;
                double2 v = make_double2(re[i][j][e], im[i][j][e]);
                if (accumulate) {
                    const double2 o = crow[col];
                    v.x += o.x;
                    v.y += o.y;
                }
                crow[col] = v;
            }
    }
}

}  // namespace

int ZGemmSchedule::check_bounds(int64_t a_size, int64_t b_size, int64_t c_size) const {
    for (const GemmGroup& g : groups) {
        if (g.m <= 0 || g.n <= 0) continue;
        if (g.c_off < 0 || g.c_off + (int64_t)(g.m - 1) * g.ldc + g.n > c_size || g.n > g.ldc)
            return set_error(DMRG_E_ARG, "complex GEMM output %lld (%dx%d, ld %d) outside %lld", (long long)g.c_off,
                             g.m, g.n, g.ldc, (long long)c_size);
        for (int ti = g.t0; ti < g.t1; ++ti) {
            const ZGemmTerm& t = terms[ti];
            if (t.k <= 0) continue;
            const int64_t ae = ta ? t.a_off + (int64_t)(t.k - 1) * t.lda + g.m : t.a_off + (int64_t)(g.m - 1) * t.lda + t.k;
            const int64_t be = tb ? t.b_off + (int64_t)(g.n - 1) * t.ldb + t.k : t.b_off + (int64_t)(t.k - 1) * t.ldb + g.n;
            if (t.a_off < 0 || ae > a_size || t.b_off < 0 || be > b_size)
                return set_error(DMRG_E_ARG, "complex GEMM operand outside its buffer");
        }
    }
    return DMRG_OK;
}

int ZGemmSchedule::finalize(cudaStream_t stream) {
    tiles.clear();
    for (int gi = 0; gi < (int)groups.size(); ++gi) {
        const GemmGroup& g = groups[gi];
        if (g.m <= 0 || g.n <= 0 || g.t1 <= g.t0) continue;
        int ks = 0;
        for (int t = g.t0; t < g.t1; ++t) ks += (terms[t].k + ZK - 1) / ZK;
        for (int m0 = 0; m0 < g.m; m0 += ZM)
            for (int n0 = 0; n0 < g.n; n0 += ZN) tiles.push_back(GemmTile{gi, m0, n0, ks});
    }
    std::stable_sort(tiles.begin(), tiles.end(), [](const GemmTile& a, const GemmTile& b) { return a.cost > b.cost; });
    DMRG_TRY(upload(d_terms, terms, stream));
    DMRG_TRY(upload(d_groups, groups, stream));
    DMRG_TRY(upload(d_tiles, tiles, stream));
    return DMRG_OK;
}

int launch_zgemm(const ZGemmSchedule& s, const double* A, const double* B, double* C, bool accumulate,
                 cudaStream_t stream) {
    if (s.tiles.empty()) return DMRG_OK;
    const int n = (int)s.tiles.size();
    const auto* a = reinterpret_cast<const double2*>(A);
    const auto* b = reinterpret_cast<const double2*>(B);
    auto* c = reinterpret_cast<double2*>(C);
    const auto* tr = s.d_terms.as<ZGemmTerm>();
    const auto* gr = s.d_groups.as<GemmGroup>();
    const auto* tl = s.d_tiles.as<GemmTile>();
    const int acc = accumulate ? 1 : 0;
    if (!s.ta && !s.tb) DMRG_LAUNCH zgemm_kernel<false, false><<<n, ZT, 0, stream>>>(a, b, c, tr, gr, tl, acc);
    else if (s.ta && !s.tb) DMRG_LAUNCH zgemm_kernel<true, false><<<n, ZT, 0, stream>>>(a, b, c, tr, gr, tl, acc);
    else if (!s.ta && s.tb) DMRG_LAUNCH zgemm_kernel<false, true><<<n, ZT, 0, stream>>>(a, b, c, tr, gr, tl, acc);
    else DMRG_LAUNCH zgemm_kernel<true, true><<<n, ZT, 0, stream>>>(a, b, c, tr, gr, tl, acc);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

}  // namespace dmrg
