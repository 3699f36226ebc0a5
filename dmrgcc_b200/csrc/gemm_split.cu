// Split-precision grouped multi-term block GEMM on the 5th-generation tensor
// cores (tcgen05, accumulators in tensor memory), on packed operand images.
//
// Arithmetic: every FP64 operand is split into two parts of a narrow format,
// x ~ hi + lo, and each product is taken as hi*hi + hi*lo + lo*hi (the lo*lo
// term is dropped) by three MMAs into an FP32 accumulator in tensor memory:
//   TF32: kind::tf32 MMAs, x rounded to FP32 first; block sums to ~1e-6;
//   BF16: kind::f16 MMAs on bf16 parts (half the bytes, twice the math rate);
//         ~16 bits per operand, block sums to ~1e-5.
// Each term's accumulator is read out and added, scaled by the term's weight,
// into FP64 registers, so the terms of a block sum accumulate in FP64.
//
// Packing (launch_pack): one CTA per image writes the hi/lo planes of one
// (panel, k slice) of an operand block in the tcgen05 canonical K-major
// no-swizzle layout (see gemm.cuh).  A GEMM stage is then one bulk copy
// (cp.async.bulk, no multicast) per plane of each operand, covering only the
// rows of the tile that hold data.
//
// Tile shape: 128 x 128 outputs, the MMA's N trimmed per tile to the block's
// columns (a multiple of 16).  A tcgen05.mma carries a fixed issue cost of
// some 60 cycles, about what a 128 x 64 x 8 TF32 product takes at full rate,
// so narrow tiles leave the tensor pipe mostly idle; at N = 128 the three
// products of a k step run at close to the pipe's rate.
//
// GEMM (persistent: one CTA per SM walks its own list of tiles, 576 threads,
// warp-specialised; stage counters and the accumulator pair run on across tiles):
//   warp 0 lane 0   producer: per stage waits the stage's "empty" barrier, arms
//                   the "full" barrier with the byte count, issues the copies;
//   warp 1 lane 0   MMA issuer: per stage waits "full", issues 2 k-substeps x 3
//                   MMAs into the term's accumulator (two 128-column accumulators
//                   alternate between terms), commits to "empty"; after a term's
//                   last stage commits to the accumulator's "full" barrier;
//   warps 2..17     epilogue: warp w reads TMEM lanes 32(w%4).. and columns
//                   32((w-2)/4)..+31: per term wait, tcgen05.ld, add w_t * value
//                   into FP64 registers, release the accumulator; finally store
//                   FP64 rows (or write the result as B-role images for the next
//                   GEMM) through a per-warp shared-memory staging buffer.
// Every wait is bounded: on a timeout a role records DMRG_E_NUMERIC in the
// status word and stops; the CTA frees its tensor memory and returns.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <map>
#include <tuple>

#include "gemm.cuh"

namespace dmrg {
namespace {

constexpr int TM = kPackRows, TN = kPackRows;
#ifndef DMRG_SPLIT_STAGES
#define DMRG_SPLIT_STAGES 6
#endif
constexpr int NSTAGE = DMRG_SPLIT_STAGES;
constexpr int STAGE_BYTES = 2 * kImage;                     // 32 KB: A image, then B image
constexpr int LBO = 128;  // bytes between the 16-byte k chunks of one 8-row core-matrix group
constexpr int SBO = 512;  // bytes between 8-row groups: a group's 4 chunks are contiguous
constexpr int PLANE = kPackRows * kPackRowBytes;            // a full hi plane in a stage; lo follows
constexpr int KSUB = kPackRowBytes / 32;                     // MMAs (32 bytes of k) per slice
#ifndef DMRG_SPLIT_EPILOGUE_WARPS
#define DMRG_SPLIT_EPILOGUE_WARPS 8
#endif
constexpr int NEPI = DMRG_SPLIT_EPILOGUE_WARPS;              // epilogue warps: 4 per TMEM lane quarter x column parts
constexpr int NT = 32 * (2 + NEPI);
constexpr int ECOLS = TN * 4 / NEPI;                         // accumulator columns per epilogue warp
// Epilogue staging per epilogue warp, 4 KB: 32 output rows x 16 doubles (16
// columns at a time), or one plane of the warp's share of one slice of an output
// image (ECOLS image rows x 64 bytes of k).
constexpr int EPI_OFF = NSTAGE * STAGE_BYTES;
constexpr int EPI_WARP_BYTES = 4096;
constexpr int BAR_OFF = EPI_OFF + NEPI * EPI_WARP_BYTES;
constexpr int SMEM_BYTES = BAR_OFF + 256;
static_assert(NEPI % 4 == 0 && ECOLS % 16 == 0 && ECOLS * NEPI == 4 * TN && TM == 128, "epilogue geometry");
static_assert(EPI_WARP_BYTES >= 32 * 16 * 8 && EPI_WARP_BYTES >= ECOLS * kPackRowBytes, "staging sizes");
constexpr uint32_t TMEM_COLS = 2 * TN;                       // two 128-column accumulators
constexpr long long kWaitLimit = 4000000;                    // try_wait polls before a wait gives up

static_assert(SMEM_BYTES <= 227 * 1024, "shared memory per CTA");
static_assert((SBO >> 4) < (1 << 14), "SBO fits the descriptor field");

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle, base offset 0, version 1.
__device__ __forceinline__ uint64_t make_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor: D = F32, A = B = TF32 (format 2) or BF16 (format 1),
// both K-major, M = 128, N = n (a multiple of 16, at most 256).
template <int FMT>
__host__ __device__ constexpr uint32_t idesc(int n) {
    return (1u << 4) | ((FMT == kFmtBF16 ? 1u : 2u) << 7) | ((FMT == kFmtBF16 ? 1u : 2u) << 10) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
}

// One MMA of 32 bytes of k (8 tf32 or 16 bf16 per row).
template <int FMT>
__device__ __forceinline__ void mma_split(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    if constexpr (FMT == kFmtBF16)
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
            "l"(a), "l"(b), "r"(id), "r"(acc)
            : "memory");
    else
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
            "l"(a), "l"(b), "r"(id), "r"(acc)
            : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(
                     smem_u32(bar)),
                 "r"(bytes)
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

// bounded wait for the completion of the phase of parity `phase`; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
    for (long long i = 0; i < kWaitLimit; ++i)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

// Bulk copy global -> shared (16-byte aligned, size multiple of 16), completing
// as transaction bytes on `bar`.  No multicast.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// TF32 rounding of an FP32 value, to nearest with ties away from zero: add half
// a unit of the 10-bit mantissa's last place to the magnitude bits, then clear
// the 13 bits below it (the sign bit is untouched, so it works on either sign).
__device__ __forceinline__ uint32_t tf32_bits(float x) { return (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u; }

__device__ __forceinline__ void split(double v, uint32_t& hi, uint32_t& lo) {
    const float f = (float)v;
    hi = tf32_bits(f);
    lo = tf32_bits(f - __uint_as_float(hi));
}

// bf16 parts (round to nearest even): hi = bf16(x), lo = bf16(x - hi)
__device__ __forceinline__ uint16_t bf16_bits(float x) {
    uint16_t r;
    asm("cvt.rn.bf16.f32 %0, %1;" : "=h"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void split_bf16(double v, uint16_t& hi, uint16_t& lo) {
    const float f = (float)v;
    hi = bf16_bits(f);
    lo = bf16_bits(f - __uint_as_float((uint32_t)hi << 16));
}

// Stores the split parts of v at (row r, k) of an image with `rows` rows per panel.
__device__ __forceinline__ void put_split(unsigned char* img, int rows, int r, int k, double v, int fmt) {
    const int plane = rows * kPackRowBytes;
    if (fmt == kFmtBF16) {
        const int kb = k * 2;
        const int off = (r >> 3) * SBO + (kb >> 4) * LBO + (r & 7) * 16 + (kb & 15);
        uint16_t h, l;
        split_bf16(v, h, l);
        *reinterpret_cast<uint16_t*>(img + off) = h;
        *reinterpret_cast<uint16_t*>(img + plane + off) = l;
    } else {
        const int kb = k * 4;
        const int off = (r >> 3) * SBO + (kb >> 4) * LBO + (r & 7) * 16 + (kb & 15);
        uint32_t h, l;
        split(v, h, l);
        *reinterpret_cast<uint32_t*>(img + off) = h;
        *reinterpret_cast<uint32_t*>(img + plane + off) = l;
    }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}

// ---- packing: one CTA (128 threads) per image ----------------------------------
__global__ void __launch_bounds__(128) pack_kernel(const PackJob* __restrict__ jobs, const PackImage* __restrict__ imgs,
                                                   const double* __restrict__ src, unsigned char* __restrict__ dst) {
    const PackImage im = imgs[blockIdx.x];
    const PackJob j = jobs[im.job];
    const int prow = panel_rows(j.rows, im.panel);  // rows of this panel's images
    const int tk = j.fmt == kFmtBF16 ? 32 : 16;     // k per slice
    unsigned char* out = dst + j.img_off + (int64_t)im.panel * j.slices * kImage + (int64_t)im.slice * 2 * prow * kPackRowBytes;
    const int r0 = im.panel * kPackRows, k0 = im.slice * tk;
    const double* s = src + j.src_off;
    for (int idx = threadIdx.x; idx < prow * tk; idx += blockDim.x) {
        // consecutive threads: consecutive k for row-major X, consecutive rows for transposed X
        const int r = j.trans ? idx % prow : idx / tk;
        const int k = j.trans ? idx / prow : idx % tk;
        double v = 0.0;
        if (r0 + r < j.rows && k0 + k < j.k)
            v = j.trans ? s[(int64_t)(k0 + k) * j.ld + (r0 + r)] : s[(int64_t)(r0 + r) * j.ld + (k0 + k)];
        put_split(out, prow, r, k, v, j.fmt);
    }
}

// ---- the GEMM ------------------------------------------------------------------
struct Bars {
    uint64_t full[NSTAGE], empty[NSTAGE], accf[2], acce[2];
    uint32_t tmem;
};
static_assert(sizeof(Bars) <= 256, "barrier block");

// MMA width of the tile at column panel pn of an n-column block: the columns
// left in the block rounded up to 16, at most TN.
__device__ __forceinline__ int mma_n(int n, int pn) { return min(TN, (n - pn * TN + 15) & ~15); }

template <int FMT>
__global__ void __launch_bounds__(NT, 1) gemm_split_kernel(const unsigned char* __restrict__ a_imgs,
                                                            const unsigned char* __restrict__ b_imgs,
                                                            double* __restrict__ C, double* __restrict__ Caux,
                                                            unsigned char* __restrict__ t_out,
                                                            const PackedTerm* __restrict__ terms,
                                                            const PackedGroup* __restrict__ groups,
                                                            const PackedTile* __restrict__ tiles,
                                                            const int* __restrict__ cta_first,
                                                            int accumulate, int out_mode, int* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char smem[];
    Bars& B = *reinterpret_cast<Bars*>(smem + BAR_OFF);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&B.tmem)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < NSTAGE; ++s) {
            mbar_init(&B.full[s], 1);
            mbar_init(&B.empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&B.accf[a], 1);
            mbar_init(&B.acce[a], NEPI);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = B.tmem;
    const int tile_begin = cta_first[blockIdx.x], tile_end = cta_first[blockIdx.x + 1];
    bool ok = true;

    if (warp == 0) {
        // ---- producer ----
        if (lane == 0) {
            int it = 0;
            for (int tt = tile_begin; tt < tile_end && ok; ++tt) {
                const PackedTile tile = tiles[tt];
                const PackedGroup g = groups[tile.group];
                // Only the image rows that hold data are copied (rounded up to a core
                // matrix of 8 rows, which the layout keeps contiguous): one bulk copy
                // per plane.  Rows left stale in shared memory feed only accumulator
                // rows (A) or columns (B) past the block, which are never stored.
                const uint32_t ca = (uint32_t)panel_rows(g.m, tile.pm) * kPackRowBytes;  // plane bytes
                const uint32_t cb = (uint32_t)panel_rows(g.n, tile.pn) * kPackRowBytes;
                const uint32_t tx = 2 * (ca + cb);
                for (int t = g.t0; t < g.t1 && ok; ++t) {
                    const PackedTerm tm = terms[t];
                    const unsigned char* a = a_imgs + tm.a_img + (int64_t)tile.pm * tm.slices * kImage;
                    const unsigned char* b = b_imgs + tm.b_img + (int64_t)tile.pn * tm.slices * kImage;
                    for (int s = 0; s < tm.slices; ++s, ++it) {
                        const int st = it % NSTAGE;
                        if (it >= NSTAGE && !mbar_wait(&B.empty[st], ((it / NSTAGE) - 1) & 1)) {
                            ok = false;
                            break;
                        }
                        unsigned char* dst = smem + st * STAGE_BYTES;
                        const unsigned char* as = a + (int64_t)s * 2 * ca;  // the panel's images: hi, lo planes
                        const unsigned char* bs = b + (int64_t)s * 2 * cb;
                        mbar_arrive_expect_tx(&B.full[st], tx);
                        bulk_g2s(dst, as, ca, &B.full[st]);
                        bulk_g2s(dst + PLANE, as + ca, ca, &B.full[st]);
                        bulk_g2s(dst + kImage, bs, cb, &B.full[st]);
                        bulk_g2s(dst + kImage + PLANE, bs + cb, cb, &B.full[st]);
                    }
                }
            }
            // Tail: nothing asynchronous may still target this CTA's shared memory
            // when it exits.  Wait until the copies of the last stages have landed
            // and until the MMAs that read them have completed and their commits
            // have arrived on the "empty" barriers (earlier stages were waited for
            // before their buffers were refilled).
            const int first = it > NSTAGE ? it - NSTAGE : 0;
            for (int j = first; j < it; ++j)
                if (!mbar_wait(&B.full[j % NSTAGE], (j / NSTAGE) & 1)) ok = false;
            for (int j = first; j < it; ++j)
                if (!mbar_wait(&B.empty[j % NSTAGE], (j / NSTAGE) & 1)) ok = false;
        }
    } else if (warp == 1) {
        // ---- MMA issuer ----
        if (lane == 0) {
            int it = 0, ti = 0;
            for (int tt = tile_begin; tt < tile_end && ok; ++tt) {
                const PackedTile tile = tiles[tt];
                const PackedGroup g = groups[tile.group];
                const uint32_t id = idesc<FMT>(mma_n(g.n, tile.pn));
                for (int t = g.t0; t < g.t1 && ok; ++t, ++ti) {
                    const int acc = ti & 1;
                    if (ti >= 2 && !mbar_wait(&B.acce[acc], ((ti >> 1) - 1) & 1)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const int slices = terms[t].slices;
                    const uint32_t d = tmem + (uint32_t)(acc * TN);
                    for (int s = 0; s < slices; ++s, ++it) {
                        const int st = it % NSTAGE;
                        if (!mbar_wait(&B.full[st], (it / NSTAGE) & 1)) {
                            ok = false;
                            break;
                        }
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        const uint32_t a_base = smem_u32(smem + st * STAGE_BYTES);
                        const uint32_t b_base = a_base + kImage;
#pragma unroll
                        for (int ks = 0; ks < KSUB; ++ks) {  // 32 bytes of k per MMA
                            const uint64_t ahi = make_smem_desc(a_base + 2 * ks * LBO, LBO, SBO);
                            const uint64_t alo = make_smem_desc(a_base + PLANE + 2 * ks * LBO, LBO, SBO);
                            const uint64_t bhi = make_smem_desc(b_base + 2 * ks * LBO, LBO, SBO);
                            const uint64_t blo = make_smem_desc(b_base + PLANE + 2 * ks * LBO, LBO, SBO);
                            mma_split<FMT>(d, ahi, bhi, id, (s > 0 || ks > 0) ? 1u : 0u);
                            mma_split<FMT>(d, ahi, blo, id, 1u);
                            mma_split<FMT>(d, alo, bhi, id, 1u);
                        }
                        mma_commit(&B.empty[st]);  // the stage's buffer is free once these MMAs are done
                    }
                    if (!ok) break;
                    mma_commit(&B.accf[acc]);      // the term's accumulator is complete
                }
            }
        }
    } else {
        // ---- epilogue: warps 2..17 ----
        const int quarter = warp & 3;                // TMEM lanes 32*quarter.. (rows of the tile)
        const int cq = (warp - 2) >> 2;              // accumulator columns cq*ECOLS..
        unsigned char* stg = smem + EPI_OFF + (warp - 2) * EPI_WARP_BYTES;
        int ti = 0;
        for (int tt = tile_begin; tt < tile_end && ok; ++tt) {
            const PackedTile tile = tiles[tt];
            const PackedGroup g = groups[tile.group];
            const bool live = cq * ECOLS < mma_n(g.n, tile.pn);  // the MMAs write this warp's columns
            double sum[ECOLS];
#pragma unroll
            for (int j = 0; j < ECOLS; ++j) sum[j] = 0.0;
            for (int t = g.t0; t < g.t1; ++t, ++ti) {
                const int acc = ti & 1;
                const bool got = mbar_wait(&B.accf[acc], (ti >> 1) & 1);
                if (!__all_sync(0xffffffffu, got)) {  // warp-uniform: tcgen05.ld below is .sync.aligned
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                if (live) {
                    const double w = terms[t].w;
#pragma unroll
                    for (int h = 0; h < ECOLS / 16; ++h) {
                        uint32_t v[16];
                        tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(acc * TN + cq * ECOLS + h * 16),
                                  v);
                        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                        for (int j = 0; j < 16; ++j) sum[h * 16 + j] += w * (double)__uint_as_float(v[j]);
                    }
                }
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(&B.acce[acc]);
            }
            if (!ok) break;
            // Output through this warp's staging buffer, so that global stores are
            // coalesced (a thread holds one output row; rows are written by the warp).
            const int r0 = tile.pm * TM + quarter * 32;      // first output row of this warp
            const int c0 = tile.pn * TN + cq * ECOLS;        // first output column of this warp
            if (out_mode == 0) {
                // staging: 32 rows x 16 doubles, element (r, c) at r*16 + (c ^ (r & 15))
                double* sd = reinterpret_cast<double*>(stg);
                double* Cb = g.cbuf ? Caux : C;
                const bool acc_out = accumulate && g.cbuf == 0;
                const int rows = min(32, g.m - r0);
                const int sub = lane >> 4, cl = lane & 15;    // lanes 0-15: even rows, 16-31: odd rows
#pragma unroll
                for (int h = 0; h < ECOLS / 16; ++h) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) sd[lane * 16 + (j ^ (lane & 15))] = sum[h * 16 + j];
                    __syncwarp();
                    const int col = c0 + h * 16 + cl;
                    if (col < g.n) {
                        double* cp = Cb + g.c_off + (int64_t)r0 * g.ldc + col;
                        if (acc_out) {
                            // the old values are loaded 8 rows at a time ahead of the
                            // stores: a load after a store through the same pointer
                            // would wait for it, one memory round trip per row
                            for (int rb = 0; rb < rows; rb += 16) {
                                double old[8];
#pragma unroll
                                for (int u = 0; u < 8; ++u) {
                                    const int r = rb + sub + 2 * u;
                                    old[u] = r < rows ? cp[(int64_t)r * g.ldc] : 0.0;
                                }
#pragma unroll
                                for (int u = 0; u < 8; ++u) {
                                    const int r = rb + sub + 2 * u;
                                    if (r < rows) cp[(int64_t)r * g.ldc] = old[u] + sd[r * 16 + (cl ^ (r & 15))];
                                }
                            }
                        } else {
                            for (int r = sub; r < rows; r += 2) cp[(int64_t)r * g.ldc] = sd[r * 16 + (cl ^ (r & 15))];
                        }
                    }
                    __syncwarp();
                }
            } else {
                // The output as B-role images of X = output^T (image rows = output
                // columns, k = output rows), zeros in the padding.  The warp's 32
                // output rows are 32 consecutive k: two TF32 slices or one BF16 slice.
                // Per pass of 16 columns the rows go through the staging buffer
                // (as above); each lane then reads one 16-byte chunk's worth of k
                // (4 TF32 or 8 BF16 values) of one image row, splits them and
                // stores the hi and lo chunks.  The 32 lanes of one store cover 8
                // image rows x 4 chunks: 512 contiguous bytes of a plane.
                constexpr int tk = FMT == kFmtBF16 ? 32 : 16;
                constexpr int kc = FMT == kFmtBF16 ? 8 : 4;          // k per 16-byte chunk
                constexpr int NIT = 32 / tk * 2;                     // (slice, 8-row group) pairs per pass
                double* sd = reinterpret_cast<double*>(stg);         // 32 rows x 16, (r, c) at r*16 + (c ^ (r & 15))
                const int prow = panel_rows(g.n, tile.pn);           // image rows of this panel
                const int j8 = lane & 7, cs = lane >> 3;             // row in an 8-row group, chunk in a slice
#pragma unroll
                for (int h = 0; h < ECOLS / 16; ++h) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) sd[lane * 16 + (j ^ (lane & 15))] = sum[h * 16 + j];
                    __syncwarp();
#pragma unroll
                    for (int it = 0; it < NIT; ++it) {
                        const int sh = it >> 1, gj = it & 1;         // slice of the warp's two (TF32), row group
                        const int jx = gj * 8 + j8;                  // column within the pass
                        const int jl = cq * ECOLS + h * 16 + jx;     // image row within the panel
                        const int slice = (r0 + sh * tk) / tk;
                        const int rk0 = sh * tk + cs * kc;           // first of this chunk's k, within the warp's rows
                        if (jl < prow && slice < g.t_slices) {
                            const bool col_ok = c0 + h * 16 + jx < g.n;
                            uint32_t hw[4], lw[4];
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                if constexpr (FMT == kFmtBF16) {
                                    uint16_t hb[2], lb[2];
#pragma unroll
                                    for (int e = 0; e < 2; ++e) {
                                        const int rk = rk0 + 2 * q + e;
                                        const double v = (col_ok && r0 + rk < g.m) ? sd[rk * 16 + (jx ^ (rk & 15))] : 0.0;
                                        split_bf16(v, hb[e], lb[e]);
                                    }
                                    hw[q] = (uint32_t)hb[0] | ((uint32_t)hb[1] << 16);
                                    lw[q] = (uint32_t)lb[0] | ((uint32_t)lb[1] << 16);
                                } else {
                                    const int rk = rk0 + q;
                                    const double v = (col_ok && r0 + rk < g.m) ? sd[rk * 16 + (jx ^ (rk & 15))] : 0.0;
                                    split(v, hw[q], lw[q]);
                                }
                            }
                            unsigned char* dst = t_out + g.t_img + (int64_t)tile.pn * g.t_slices * kImage +
                                                 (int64_t)slice * 2 * prow * kPackRowBytes + (jl >> 3) * SBO + cs * LBO +
                                                 j8 * 16;
                            *reinterpret_cast<uint4*>(dst) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                            *reinterpret_cast<uint4*>(dst + prow * kPackRowBytes) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
                        }
                    }
                    __syncwarp();
                }
            }
        }
    }
    __syncwarp();  // producer and MMA warps: lanes 1..31 wait for lane 0
    if (!ok) atomicExch(status, DMRG_E_NUMERIC);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// Deterministic split-K reduction (the scheme of gemm_f64.cu): chunks summed in order.
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

}  // namespace

int64_t PackSchedule::add(int64_t src_off, int rows, int k, int ld, bool trans) {
    const int tk = pack_k(fmt);
    PackJob j{};
    j.fmt = fmt;
    j.src_off = src_off;
    j.img_off = bytes;
    j.rows = rows;
    j.k = k;
    j.ld = ld;
    j.trans = trans ? 1 : 0;
    j.slices = (k + tk - 1) / tk;
    const int panels = (rows + kPackRows - 1) / kPackRows;
    const int job = (int)jobs.size();
    jobs.push_back(j);
    for (int p = 0; p < panels; ++p)
        for (int s = 0; s < j.slices; ++s) images.push_back(PackImage{job, p, s, 0});
    bytes += image_bytes(rows, j.slices);
    return j.img_off;
}

int PackSchedule::finalize(cudaStream_t stream) {
    DMRG_TRY(upload(d_jobs, jobs, stream));
    DMRG_TRY(upload(d_images, images, stream));
    return DMRG_OK;
}

int launch_pack(const PackSchedule& p, const double* src, unsigned char* dst, cudaStream_t stream) {
    if (p.images.empty()) return DMRG_OK;
    DMRG_LAUNCH pack_kernel<<<(int)p.images.size(), 128, 0, stream>>>(p.d_jobs.as<PackJob>(), p.d_images.as<PackImage>(), src,
                                                          dst);
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

int prepare_split_kernel(int fmt);  // below: the kernel's shared-memory opt-in on this device

int PackedSchedule::finalize(cudaStream_t stream, int num_sms) {
    DMRG_TRY(prepare_split_kernel(fmt));
    exec_groups.clear();
    splits.clear();
    tiles.clear();
    aux_size = 0;
    auto stages = [&](const PackedGroup& g) {
        int64_t s = 0;
        for (int t = g.t0; t < g.t1; ++t) s += terms[t].slices;
        return s;
    };
    int64_t total = 0;
    for (const PackedGroup& g : groups)
        total += stages(g) * ((g.m + TM - 1) / TM) * ((g.n + TN - 1) / TN);
    const int64_t share = (num_sms > 0 && out_mode == 0) ? std::max<int64_t>(8, total / ((int64_t)num_sms * 2)) : 0;
    for (const PackedGroup& g : groups) {
        if (g.m <= 0 || g.n <= 0 || g.t1 <= g.t0) continue;
        const int64_t st = stages(g);
        if (share == 0 || st <= 2 * share || g.t1 - g.t0 < 2) {
            exec_groups.push_back(g);
            continue;
        }
        GemmSplit sp{g.c_off, aux_size, g.ldc, g.m, g.n, 0};
        int t0 = g.t0;
        int64_t acc = 0;
        for (int t = g.t0; t < g.t1; ++t) {
            acc += terms[t].slices;
            if (acc >= share || t + 1 == g.t1) {
                PackedGroup c = g;
                c.t0 = t0;
                c.t1 = t + 1;
                c.c_off = aux_size + (int64_t)sp.chunks * g.m * g.n;
                c.ldc = g.n;
                c.cbuf = 1;
                exec_groups.push_back(c);
                sp.chunks++;
                t0 = t + 1;
                acc = 0;
            }
        }
        aux_size += (int64_t)sp.chunks * g.m * g.n;
        splits.push_back(sp);
    }
    // Tile cost in quarter stages: 4 per stage (its MMAs), 1 per term (the
    // accumulator read-out), 6 per tile (pipeline fill and the output store).
    std::vector<PackedTile> all;
    for (int gi = 0; gi < (int)exec_groups.size(); ++gi) {
        const PackedGroup& g = exec_groups[gi];
        const int cost = (int)(4 * stages(g) + (g.t1 - g.t0) + 6);
        for (int pm = 0; pm * TM < g.m; ++pm)
            for (int pn = 0; pn * TN < g.n; ++pn) all.push_back(PackedTile{gi, pm, pn, cost});
    }
    std::stable_sort(all.begin(), all.end(), [](const PackedTile& a, const PackedTile& b) { return a.cost > b.cost; });
    // Longest-processing-time-first assignment to the persistent CTAs: each
    // tile, heaviest first, goes to the least loaded CTA (lowest index on ties).
    // A CTA's tiles are stored contiguously, heaviest first.
    ctas = (int)std::min<int64_t>((int64_t)all.size(), num_sms > 0 ? num_sms : 148);
    std::vector<int> owner(all.size());
    std::vector<int> count(std::max(ctas, 1), 0);
    {
        std::vector<std::pair<int64_t, int>> heap;
        for (int c = 0; c < ctas; ++c) heap.push_back({0, c});
        auto later = [](const std::pair<int64_t, int>& a, const std::pair<int64_t, int>& b) { return a > b; };
        for (size_t i = 0; i < all.size(); ++i) {
            std::pop_heap(heap.begin(), heap.end(), later);
            auto& least = heap.back();
            least.first += all[i].cost;
            owner[i] = least.second;
            count[least.second]++;
            std::push_heap(heap.begin(), heap.end(), later);
        }
    }
    cta_first.assign(ctas + 1, 0);
    for (int c = 0; c < ctas; ++c) cta_first[c + 1] = cta_first[c] + count[c];
    tiles.resize(all.size());
    {
        std::vector<int> next(cta_first.begin(), cta_first.end() - 1);
        for (size_t i = 0; i < all.size(); ++i) tiles[next[owner[i]]++] = all[i];
    }
    DMRG_TRY(upload(d_terms, terms, stream));
    DMRG_TRY(upload(d_groups, exec_groups, stream));
    DMRG_TRY(upload(d_tiles, tiles, stream));
    DMRG_TRY(upload(d_cta_first, cta_first, stream));
    DMRG_TRY(upload(d_splits, splits, stream));
    DMRG_TRY(aux.alloc((size_t)std::max<int64_t>(aux_size, 1) * sizeof(double)));
    return DMRG_OK;
}

int PackedSchedule::check_bounds(int64_t a_bytes, int64_t b_bytes, int64_t c_size, int64_t t_bytes) const {
    for (const PackedGroup& g : groups) {
        if (g.m <= 0 || g.n <= 0) continue;
        for (int t = g.t0; t < g.t1; ++t) {
            const PackedTerm& tm = terms[t];
            if (tm.a_img < 0 || tm.a_img + image_bytes(g.m, tm.slices) > a_bytes || tm.b_img < 0 ||
                tm.b_img + image_bytes(g.n, tm.slices) > b_bytes || tm.a_img % 16 || tm.b_img % 16)
                return set_error(DMRG_E_ARG, "packed GEMM term %d reads outside its images", t);
        }
        if (out_mode == 0) {
            if (g.c_off < 0 || g.c_off + (int64_t)(g.m - 1) * g.ldc + g.n > c_size || g.n > g.ldc)
                return set_error(DMRG_E_ARG, "packed GEMM output %lld outside %lld", (long long)g.c_off,
                                 (long long)c_size);
        } else if (g.t_img < 0 || g.t_img + image_bytes(g.n, g.t_slices) > t_bytes ||
                   (int64_t)g.t_slices * pack_k(fmt) < g.m || g.t_img % 16) {
            return set_error(DMRG_E_ARG, "packed GEMM output images outside their buffer");
        }
    }
    return DMRG_OK;
}

namespace {
// The kernel's dynamic shared-memory opt-in, once per device and format.  It is
// made when a schedule is finalized (operator creation), so that no launch
// inside a stream capture (the graph-captured Lanczos loop) has to make it.
std::atomic<bool> g_smem_attr[2][64];
template <int FMT>
int ensure_smem_attr() {
    int dev = 0;
    DMRG_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(DMRG_E_ARG, "device ordinal %d not supported", dev);
    if (!g_smem_attr[FMT][dev].load()) {
        DMRG_CUDA_TRY(
            cudaFuncSetAttribute(gemm_split_kernel<FMT>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
        g_smem_attr[FMT][dev].store(true);
    }
    return DMRG_OK;
}

template <int FMT>
int launch_fmt(const PackedSchedule& s, const unsigned char* a_imgs, const unsigned char* b_imgs, double* C,
               unsigned char* t_out, bool accumulate, int* status, int grid, cudaStream_t stream) {
    DMRG_TRY(ensure_smem_attr<FMT>());
    DMRG_LAUNCH gemm_split_kernel<FMT><<<grid, NT, SMEM_BYTES, stream>>>(
        a_imgs, b_imgs, C, s.aux.as<double>(), t_out, s.d_terms.as<PackedTerm>(), s.d_groups.as<PackedGroup>(),
        s.d_tiles.as<PackedTile>(), s.d_cta_first.as<int>(), accumulate ? 1 : 0, s.out_mode, status);
    return DMRG_OK;
}
}  // namespace

int prepare_split_kernel(int fmt) {
    return fmt == kFmtBF16 ? ensure_smem_attr<kFmtBF16>() : ensure_smem_attr<kFmtTF32>();
}

int launch_gemm_split(const PackedSchedule& s, const unsigned char* a_imgs, const unsigned char* b_imgs, double* C,
                      unsigned char* t_out, bool accumulate, int* status, cudaStream_t stream) {
    if (s.tiles.empty()) return DMRG_OK;
    // persistent: one CTA per SM walks its own run of tiles (assigned at
    // finalize); its stage ring and accumulator pair carry over from one tile
    // to the next
    const int grid = s.ctas;
    if (s.fmt == kFmtBF16) DMRG_TRY(launch_fmt<kFmtBF16>(s, a_imgs, b_imgs, C, t_out, accumulate, status, grid, stream));
    else DMRG_TRY(launch_fmt<kFmtTF32>(s, a_imgs, b_imgs, C, t_out, accumulate, status, grid, stream));
    if (!s.splits.empty()) {
        int64_t biggest = 0;
        for (const GemmSplit& sp : s.splits) biggest = std::max<int64_t>(biggest, (int64_t)sp.m * sp.n);
        const int gx = (int)std::min<int64_t>((biggest + 255) / 256, 64);
        DMRG_LAUNCH split_reduce_tf32_kernel<<<dim3(gx, (unsigned)s.splits.size()), 256, 0, stream>>>(
            C, s.aux.as<double>(), s.d_splits.as<GemmSplit>(), accumulate ? 1 : 0);
    }
    DMRG_CUDA_TRY(cudaGetLastError());
    return DMRG_OK;
}

}  // namespace dmrg

namespace dmrg {

int SplitPlan::build(const GemmSchedule& s, int fmt, int64_t a_size, int64_t b_size, int64_t c_size, cudaStream_t st,
                     int num_sms) {
    pa = PackSchedule();
    pb = PackSchedule();
    ps.reset();
    pa.fmt = pb.fmt = ps.fmt = fmt;
    ps.out_mode = 0;
    const int tk = pack_k(fmt);
    // one image per distinct operand block (the same block often serves many terms)
    std::map<std::tuple<int64_t, int, int, int>, int64_t> a_img, b_img;
    for (const GemmGroup& g : s.groups) {
        if (g.m <= 0 || g.n <= 0 || g.t1 <= g.t0) continue;
        PackedGroup pg{};
        pg.t0 = (int)ps.terms.size();
        pg.m = g.m;
        pg.n = g.n;
        pg.c_off = g.c_off;
        pg.ldc = g.ldc;
        for (int t = g.t0; t < g.t1; ++t) {
            const GemmTerm& x = s.terms[t];
            if (x.k <= 0) continue;
            // A role: X = op(A), m x k;  B role: X = op(B)^T, n x k
            const auto ka = std::make_tuple(x.a_off, g.m, x.k, x.lda);
            auto ia = a_img.find(ka);
            if (ia == a_img.end()) ia = a_img.emplace(ka, pa.add(x.a_off, g.m, x.k, x.lda, s.ta)).first;
            const auto kb = std::make_tuple(x.b_off, g.n, x.k, x.ldb);
            auto ib = b_img.find(kb);
            if (ib == b_img.end()) ib = b_img.emplace(kb, pb.add(x.b_off, g.n, x.k, x.ldb, !s.tb)).first;
            ps.terms.push_back(PackedTerm{ia->second, ib->second, (x.k + tk - 1) / tk, 0, x.scale});
        }
        pg.t1 = (int)ps.terms.size();
        if (pg.t1 > pg.t0) ps.groups.push_back(pg);
    }
    // every packed operand inside its source buffer
    for (const PackJob& j : pa.jobs) {
        const int64_t end = j.trans ? j.src_off + (int64_t)(j.k - 1) * j.ld + j.rows
                                    : j.src_off + (int64_t)(j.rows - 1) * j.ld + j.k;
        if (j.src_off < 0 || end > a_size) return set_error(DMRG_E_ARG, "split plan: A operand outside its buffer");
    }
    for (const PackJob& j : pb.jobs) {
        const int64_t end = j.trans ? j.src_off + (int64_t)(j.k - 1) * j.ld + j.rows
                                    : j.src_off + (int64_t)(j.rows - 1) * j.ld + j.k;
        if (j.src_off < 0 || end > b_size) return set_error(DMRG_E_ARG, "split plan: B operand outside its buffer");
    }
    DMRG_TRY(ps.check_bounds(pa.bytes, pb.bytes, c_size, 0));
    DMRG_TRY(pa.finalize(st));
    DMRG_TRY(pb.finalize(st));
    DMRG_TRY(ps.finalize(st, num_sms));
    DMRG_TRY(img_a.alloc((size_t)std::max<int64_t>(pa.bytes, 16)));
    DMRG_TRY(img_b.alloc((size_t)std::max<int64_t>(pb.bytes, 16)));
    return DMRG_OK;
}

int SplitPlan::run(const double* A, const double* B, double* C, bool accumulate, int* status,
                   cudaStream_t st) const {
    DMRG_TRY(launch_pack(pa, A, img_a.as<unsigned char>(), st));
    DMRG_TRY(launch_pack(pb, B, img_b.as<unsigned char>(), st));
    return launch_gemm_split(ps, img_a.as<unsigned char>(), img_b.as<unsigned char>(), C, nullptr, accumulate,
                             status, st);
}

}  // namespace dmrg
