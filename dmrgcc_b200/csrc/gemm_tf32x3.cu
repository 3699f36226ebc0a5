// Split-precision grouped multi-term block GEMM on the 5th-generation tensor
// cores (tcgen05, accumulators in tensor memory): the same schedules as
// gemm_f64.cu, with every FP64 operand rounded to FP32 and split on the fly into
// two TF32 parts, x ~ hi + lo, and each product taken as hi*hi + hi*lo + lo*hi
// (the lo*lo term, ~2^-22 relative, is dropped), accumulated in FP32 in TMEM and
// stored as FP64.  Relative error of a block sum ~1e-6.
//
// CTA: 128 threads, output tile 128 x 64 (tcgen05.mma M=128, N=64, K=8 per
// instruction), k-step 32 per stage, two stages.  All threads load the FP64
// operands (four consecutive K values per thread), scale A by the term's
// weight, split, and store hi and lo planes in shared memory in the canonical
// K-major no-swizzle layout: core matrices of 8 rows x 16 bytes, 8-row groups
// 128 bytes apart (SBO), 16-byte K chunks LBO apart; LBO carries a 16-byte pad
// so that the 16-byte stores of consecutive threads hit distinct banks.  One
// thread issues the stage's 12 MMAs (4 k-substeps x 3 products) and commits
// them to the stage's mbarrier; a stage is refilled only after that barrier
// completes.  Epilogue: warp w reads TMEM lanes 32w..32w+31 (= tile rows) with
// tcgen05.ld and writes or adds the FP64 results.
// Every wait is bounded: on a timeout the kernel records DMRG_E_NUMERIC in the
// status word, waits (bounded again) for its MMAs in flight, frees its TMEM and
// returns; the decision to stop is block-uniform.
#include <algorithm>
#include <cstdint>

#include "gemm.cuh"

namespace dmrg {
namespace {

constexpr int TM = 128, TN = 64, TK = 32, NT = 128;
constexpr int CHUNKS = TK / 4;               // 16-byte K chunks per stage (4 tf32 each)
constexpr int LBO_A = TM * 16 + 16;          // bytes between K chunks of A (padded)
constexpr int LBO_B = TN * 16 + 16;
constexpr int SBO = 128;                     // bytes between 8-row core-matrix groups
constexpr int PLANE_A = CHUNKS * LBO_A;      // one of hi / lo
constexpr int PLANE_B = CHUNKS * LBO_B;
constexpr int STAGE_BYTES = 2 * PLANE_A + 2 * PLANE_B;
constexpr int SMEM_BYTES = 2 * STAGE_BYTES + 64;
constexpr uint32_t TMEM_COLS = 64;
constexpr long long kWaitLimit = 4000000;    // try_wait polls before a wait gives up

static_assert(LBO_A % 16 == 0 && LBO_B % 16 == 0 && STAGE_BYTES % 16 == 0, "16-byte descriptor units");
static_assert((LBO_A >> 4) < (1 << 14) && (LBO_B >> 4) < (1 << 14), "LBO fits the descriptor field");

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle, base offset 0, version 1.
__device__ __forceinline__ uint64_t make_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor: D = F32, A = B = TF32, both K-major, N = 64, M = 128.
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TN >> 3) << 17) |
                           ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(IDESC), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// bounded wait for the completion of phase `phase`; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
    for (long long i = 0; i < kWaitLimit; ++i)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

__device__ __forceinline__ uint32_t tf32_bits(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void split(double v, uint32_t& hi, uint32_t& lo) {
    const float f = (float)v;
    hi = tf32_bits(f);
    lo = tf32_bits(f - __uint_as_float(hi));
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}

// One stage: A (TM x TK, scaled by the term weight) and B (TN x TK), K-major planes.
template <bool TA, bool TB>
__device__ __forceinline__ void fill_stage(unsigned char* st, const double* __restrict__ A,
                                           const double* __restrict__ B, const GemmTerm& t, int k0, int m0, int n0,
                                           int m, int n, int tid) {
    unsigned char* a_hi = st;
    unsigned char* a_lo = st + PLANE_A;
    unsigned char* b_hi = st + 2 * PLANE_A;
    unsigned char* b_lo = b_hi + PLANE_B;
    const double scale = t.scale;
#pragma unroll 2
    for (int idx = tid; idx < TM * CHUNKS; idx += NT) {
        const int r = TA ? (idx % TM) : (idx / CHUNKS);
        const int c = TA ? (idx / TM) : (idx % CHUNKS);
        uint32_t h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int k = k0 + 4 * c + e;
            double v = 0.0;
            if (m0 + r < m && k < t.k)
                v = TA ? A[t.a_off + (int64_t)k * t.lda + (m0 + r)] : A[t.a_off + (int64_t)(m0 + r) * t.lda + k];
            split(v * scale, h[e], l[e]);
        }
        const int off = c * LBO_A + (r >> 3) * SBO + (r & 7) * 16;
        *reinterpret_cast<uint4*>(a_hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(a_lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
#pragma unroll 2
    for (int idx = tid; idx < TN * CHUNKS; idx += NT) {
        const int r = TB ? (idx / CHUNKS) : (idx % TN);
        const int c = TB ? (idx % CHUNKS) : (idx / TN);
        uint32_t h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int k = k0 + 4 * c + e;
            double v = 0.0;
            if (n0 + r < n && k < t.k)
                v = TB ? B[t.b_off + (int64_t)(n0 + r) * t.ldb + k] : B[t.b_off + (int64_t)k * t.ldb + (n0 + r)];
            split(v, h[e], l[e]);
        }
        const int off = c * LBO_B + (r >> 3) * SBO + (r & 7) * 16;
        *reinterpret_cast<uint4*>(b_hi + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4*>(b_lo + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(NT) gemm_tf32x3_kernel(const double* __restrict__ A, const double* __restrict__ B,
                                                         double* __restrict__ C, double* __restrict__ Caux,
                                                         const GemmTerm* __restrict__ terms,
                                                         const GemmGroup* __restrict__ groups,
                                                         const GemmTile* __restrict__ tiles, int accumulate,
                                                         int* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* stage_mem[2] = {smem, smem + STAGE_BYTES};
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * STAGE_BYTES);          // 2 stage barriers
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + 2 * STAGE_BYTES + 32);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const GemmTile tile = tiles[blockIdx.x];
    const GemmGroup g = groups[tile.group];

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[0])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[1])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    bool ok = true;
    int issued = 0;              // stages committed so far
    uint32_t phase[2] = {0, 0};  // parity of the next completion to wait for, per stage
    int t = g.t0, k0 = 0;
    GemmTerm cur = terms[t];
    while (t < g.t1) {
        const int s = issued & 1;
        bool mine = true;
        if (issued >= 2) {  // the MMAs that last read this stage must be done
            mine = mbar_wait(&bars[s], phase[s]);
            phase[s] ^= 1u;
        }
        if (mine) fill_stage<TA, TB>(stage_mem[s], A, B, cur, k0, tile.m0, tile.n0, g.m, g.n, tid);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        if (!__syncthreads_and(mine ? 1 : 0)) {
            ok = false;
            break;
        }
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a_base = smem_u32(stage_mem[s]);
            const uint32_t b_base = a_base + 2 * PLANE_A;
#pragma unroll
            for (int ks = 0; ks < TK / 8; ++ks) {
                const uint64_t ahi = make_smem_desc(a_base + 2 * ks * LBO_A, LBO_A, SBO);
                const uint64_t alo = make_smem_desc(a_base + PLANE_A + 2 * ks * LBO_A, LBO_A, SBO);
                const uint64_t bhi = make_smem_desc(b_base + 2 * ks * LBO_B, LBO_B, SBO);
                const uint64_t blo = make_smem_desc(b_base + PLANE_B + 2 * ks * LBO_B, LBO_B, SBO);
                mma_tf32(tmem, ahi, bhi, (issued > 0 || ks > 0) ? 1u : 0u);
                mma_tf32(tmem, ahi, blo, 1u);
                mma_tf32(tmem, alo, bhi, 1u);
            }
            mma_commit(&bars[s]);
        }
        ++issued;
        k0 += TK;
        if (k0 >= cur.k) {
            k0 = 0;
            ++t;
            if (t < g.t1) cur = terms[t];
        }
    }
    // every commit not yet waited for (the last one or two stages) must complete,
    // on the error path too, before TMEM is read or freed
    bool drained = true;
    for (int j = 0; j < 2 && j < issued; ++j) {
        const int st_idx = (issued - 1 - j) & 1;
        if (!mbar_wait(&bars[st_idx], phase[st_idx])) drained = false;
    }
    ok = __syncthreads_and((ok && drained) ? 1 : 0) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok && issued > 0) {
        const bool acc_out = accumulate && g.cbuf == 0;
        double* Cb = g.cbuf ? Caux : C;
        const int row = tile.m0 + warp * 32 + lane;
#pragma unroll
        for (int half = 0; half < TN / 32; ++half) {
            uint32_t v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(half * 32), v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < g.m) {
                double* crow = Cb + g.c_off + (int64_t)row * g.ldc;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int col = tile.n0 + half * 32 + j;
                    if (col < g.n) {
                        const double x = (double)__uint_as_float(v[j]);
                        crow[col] = acc_out ? crow[col] + x : x;
                    }
                }
            }
        }
    }
    if (!ok && tid == 0) atomicExch(status, DMRG_E_NUMERIC);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// Deterministic split-K reduction (the same scheme as gemm_f64.cu): grid (element
// slices, split groups), chunks summed in a fixed order.
__global__ void __launch_bounds__(256) split_reduce_tf32_kernel(double* __restrict__ C,
                                                                const double* __restrict__ Caux,
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

template <bool TA, bool TB>
int launch_variant(const GemmSchedule& s, const double* A, const double* B, double* C, bool accumulate, int* status,
                   cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
        DMRG_CUDA_TRY(cudaFuncSetAttribute(gemm_tf32x3_kernel<TA, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           SMEM_BYTES));
        attr = true;
    }
    gemm_tf32x3_kernel<TA, TB><<<(int)s.tiles.size(), NT, SMEM_BYTES, st>>>(
        A, B, C, s.aux.as<double>(), s.d_terms.as<GemmTerm>(), s.d_groups.as<GemmGroup>(), s.d_tiles.as<GemmTile>(),
        accumulate ? 1 : 0, status);
    return DMRG_OK;
}

}  // namespace

int launch_gemm_tf32x3(const GemmSchedule& s, const double* A, const double* B, double* C, bool accumulate,
                       int* status, cudaStream_t stream) {
    if (s.tiles.empty()) return DMRG_OK;
    if (s.tile_m != TM || s.tile_n != TN)
        return set_error(DMRG_E_ARG, "TF32X3 GEMM needs a %dx%d tile schedule (got %dx%d)", TM, TN, s.tile_m, s.tile_n);
    if (!s.ta && !s.tb) DMRG_TRY((launch_variant<false, false>(s, A, B, C, accumulate, status, stream)));
    else if (s.ta && !s.tb) DMRG_TRY((launch_variant<true, false>(s, A, B, C, accumulate, status, stream)));
    else if (!s.ta && s.tb) DMRG_TRY((launch_variant<false, true>(s, A, B, C, accumulate, status, stream)));
    else DMRG_TRY((launch_variant<true, true>(s, A, B, C, accumulate, status, stream)));
    if (!s.splits.empty()) {
        int64_t biggest = 0;
        for (const GemmSplit& sp : s.splits) biggest = std::max<int64_t>(biggest, (int64_t)sp.m * sp.n);
        const int gx = (int)std::min<int64_t>((biggest + 255) / 256, 64);
        split_reduce_tf32_kernel<<<dim3(gx, (unsigned)s.splits.size()), 256, 0, stream>>>(
            C, s.aux.as<double>(), s.d_splits.as<GemmSplit>(), accumulate ? 1 : 0);
    }
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

}  // namespace dmrg
