// Grouped multi-term block GEMM: the one contraction engine behind H_eff*psi,
// the environment updates and the merge.
//
// A launch processes a list of output blocks ("groups").  Group g owns a
// row-major m x n block C_g at C + c_off (leading dimension ldc) and a range of
// terms [t0, t1); each term contributes scale * op(A_t) @ op(B_t) with A_t at
// A + a_off (m x k, or k x m when TA) and B_t at B + b_off (k x n, or n x k when
// TB).  All terms of a group are summed in registers by the CTA that owns the
// output tile, so no atomics are needed and the summation order is fixed.
// Work items ("tiles") are (group, m0, n0) output tiles, sorted by cost.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace dmrg {

struct GemmTerm {
    int64_t a_off;
    int64_t b_off;
    int lda;
    int ldb;
    int k;
    int pad_;
    double scale;
};

struct GemmGroup {
    int64_t c_off;
    int ldc;
    int m;
    int n;
    int t0;
    int t1;
    int cbuf;  // 0: output goes to C; 1: a split-K chunk, output goes to the schedule's aux buffer
};

// A group whose term list was split into chunks: aux holds `chunks` consecutive
// m x n partial tiles that are summed, in chunk order, into C at c_off.
struct GemmSplit {
    int64_t c_off;
    int64_t aux_off;
    int ldc;
    int m;
    int n;
    int chunks;
};

struct GemmTile {
    int group;
    int m0;
    int n0;
    int cost;  // k-steps, used for ordering only
};

// Host-side schedule of one launch.
struct GemmSchedule {
    std::vector<GemmTerm> terms;
    std::vector<GemmGroup> groups;
    std::vector<GemmTile> tiles;
    bool ta = false, tb = false;
    double flops = 0.0;  // 2*m*n*k summed over terms
    // execution form built by finalize(): split-K chunks replace long groups
    std::vector<GemmGroup> exec_groups;
    std::vector<GemmSplit> splits;
    int64_t aux_size = 0;
    int tile_m = 0, tile_n = 0, tile_k = 0;  // set by finalize()
    // device copies
    DeviceBuffer d_terms, d_groups, d_tiles, d_splits, aux;

    void reset() {
        terms.clear();
        groups.clear();
        tiles.clear();
        ta = tb = false;
        flops = 0.0;
        exec_groups.clear();
        splits.clear();
        aux_size = 0;
    }
    int add_group(int64_t c_off, int ldc, int m, int n) {
        GemmGroup g{c_off, ldc, m, n, (int)terms.size(), (int)terms.size(), 0};
        groups.push_back(g);
        return (int)groups.size() - 1;
    }
    // Terms must be appended to the most recently added group.
    void add_term(int64_t a_off, int lda, int64_t b_off, int ldb, int k, double scale) {
        GemmGroup& g = groups.back();
        terms.push_back(GemmTerm{a_off, b_off, lda, ldb, k, 0, scale});
        g.t1 = (int)terms.size();
        flops += 2.0 * g.m * g.n * (double)k;
    }
    // Verifies that every read of A/B and every write of C stays inside buffers
    // of the given sizes (doubles); returns DMRG_E_ARG (no launch) otherwise.
    int check_bounds(int64_t a_size, int64_t b_size, int64_t c_size) const;
    // Builds the tile list (tile_m x tile_n tiles, heaviest first) and uploads.
    // With `num_sms` > 0, groups whose k-loop is much longer than the balanced
    // per-CTA share are split into chunks (split-K) reduced by a second kernel,
    // so that a few very long output tiles do not leave the GPU idle.
    int finalize(int tile_m, int tile_n, int tile_k, cudaStream_t stream, int num_sms = 0);
};

// C (+)= sum of terms for every tile of `s`.  A, B, C are the base pointers.
int launch_gemm_f64(const GemmSchedule& s, const double* A, const double* B, double* C,
                    bool accumulate, cudaStream_t stream);

// ---------------------------------------------------------------------------
// Split-precision paths on the tcgen05 tensor cores (gemm_split.cu).
//
// Operands are packed once into "images": for an operand block X (rows x k,
// K-major), image (panel p, slice s) holds rows [p*R, p*R+R) x one k slice as a
// hi plane followed by a lo plane (x ~ hi + lo), each in the tcgen05 canonical
// K-major no-swizzle layout: 64 bytes of k per row in 16-byte chunks; a core
// matrix is 8 rows x 16 bytes, the 4 chunks of an 8-row group are contiguous
// (LBO = 128) and groups follow each other (SBO = 512), so the first m rows of
// a plane are one contiguous prefix: byte offset of (row r, k) =
// (r/8)*512 + (k*E/16)*128 + (r%8)*16 + (k*E)%16 for E-byte elements.  Zero
// outside X.  Two formats share this geometry:
//   TF32 (E = 4): x rounded to FP32, hi = tf32(x), lo = tf32(x - hi); 16 k per slice;
//   BF16 (E = 2): hi = bf16(x), lo = bf16(x - hi); 32 k per slice.
// R = 128 rows per panel in both roles (A: output rows, B: output columns),
// except the last panel of a block, which keeps only the block's remaining rows
// rounded up to a core matrix of 8 (its images are that much shorter).  The
// images of panel p follow those of the full panels before it, slice by slice.
// A GEMM stage then is one contiguous bulk copy per plane of each operand.
constexpr int kFmtTF32 = 0, kFmtBF16 = 1;
constexpr int kPackRowBytes = 64;
constexpr int kPackRows = 128;
constexpr int kImage = 2 * kPackRows * kPackRowBytes;  // bytes of a full image: hi + lo
inline int pack_k(int fmt) { return fmt == kFmtBF16 ? 32 : 16; }  // k per slice
// rows held by panel p of a block of `rows` rows
__host__ __device__ inline int panel_rows(int rows, int p) {
    const int r = (rows - p * kPackRows + 7) & ~7;
    return r < kPackRows ? r : kPackRows;
}
// bytes of all images of a block of `rows` rows and `slices` k slices
inline int64_t image_bytes(int rows, int slices) {
    const int64_t full = rows / kPackRows, rest = rows - full * kPackRows;
    return (full * kPackRows + ((rest + 7) & ~7)) * 2 * kPackRowBytes * slices;
}

struct PackJob {
    int64_t src_off;  // doubles
    int64_t img_off;  // bytes, into the image buffer
    int rows, k, ld;  // logical X: rows x k; X(r, c) = src[src_off + (trans ? c*ld + r : r*ld + c)]
    int trans;
    int prow_;
    int slices;       // ceil(k / pack_k(fmt))
    int fmt;          // kFmtTF32 or kFmtBF16
    int pad_;
};
struct PackImage {
    int job, panel, slice, pad_;
};
struct PackSchedule {
    int fmt = kFmtTF32;
    std::vector<PackJob> jobs;
    std::vector<PackImage> images;
    int64_t bytes = 0;
    DeviceBuffer d_jobs, d_images;
    // Appends the images of one operand block; returns its image offset (bytes).
    int64_t add(int64_t src_off, int rows, int k, int ld, bool trans);
    int finalize(cudaStream_t stream);
};
// dst (images) <- split-precision images of the jobs' blocks of src.
int launch_pack(const PackSchedule& p, const double* src, unsigned char* dst, cudaStream_t stream);

struct PackedTerm {
    int64_t a_img, b_img;  // image offsets (bytes) of the A operand (A role) and the B operand (B role)
    int slices;            // ceil(k / pack_k(fmt)), the same for both
    int pad_;
    double w;              // weight of this product
};
struct PackedGroup {
    int t0, t1;            // terms
    int m, n;              // output block
    int64_t c_off;         // output mode 0: FP64 block at C + c_off (ldc), or its split-K chunk in aux
    int ldc;
    int cbuf;              // 1: split-K chunk, written to aux
    int64_t t_img;         // output mode 1: the output written as B-role images (rows = columns n,
    int t_slices;          // k = rows m) for a following packed GEMM; t_slices = ceil(m / pack_k(fmt))
    int pad_;
};
struct PackedTile {
    int group, pm, pn, cost;
};
struct PackedSchedule {
    int fmt = kFmtTF32;
    std::vector<PackedTerm> terms;
    std::vector<PackedGroup> groups;
    int out_mode = 0;  // 0: FP64 output blocks, 1: B-role images
    std::vector<PackedGroup> exec_groups;
    std::vector<GemmSplit> splits;
    std::vector<PackedTile> tiles;  // grouped by persistent CTA
    std::vector<int> cta_first;     // CTA c runs tiles [cta_first[c], cta_first[c + 1])
    int ctas = 0;                   // grid of the persistent launch
    int64_t aux_size = 0;
    DeviceBuffer d_terms, d_groups, d_tiles, d_cta_first, d_splits, aux;
    void reset() {
        terms.clear();
        groups.clear();
        exec_groups.clear();
        splits.clear();
        tiles.clear();
        cta_first.clear();
        ctas = 0;
        aux_size = 0;
    }
    // Verifies every image read and every output write against the buffer sizes
    // (bytes for images, doubles for c_size); DMRG_E_ARG, no launch, otherwise.
    int check_bounds(int64_t a_bytes, int64_t b_bytes, int64_t c_size, int64_t t_bytes) const;
    // Splits long mode-0 groups (num_sms > 0), builds the 128 x 128 tiles and
    // assigns them to min(tiles, num_sms or 148) persistent CTAs by cost
    // (longest first, to the least loaded CTA), uploads.
    int finalize(cudaStream_t stream, int num_sms = 0);
};
// C (+)= the products of every group (mode 0), or t_out <- images of them (mode 1),
// in the schedule's format.  A wait that gives up sets *status = DMRG_E_NUMERIC.
int launch_gemm_split(const PackedSchedule& s, const unsigned char* a_imgs, const unsigned char* b_imgs,
                       double* C, unsigned char* t_out, bool accumulate, int* status, cudaStream_t stream);

// Any FP64 grouped GEMM schedule run in split precision: every distinct A
// operand block becomes an A-role image, every distinct B operand block a
// B-role image (its transpose, K-major), and each group's terms accumulate in
// FP32 tensor memory per term and in FP64 across terms (mode-0 output).
struct SplitPlan {
    PackSchedule pa, pb;
    PackedSchedule ps;
    DeviceBuffer img_a, img_b;
    // Builds the plan for `s` (its groups, terms and transposes) in format fmt
    // (kFmtTF32 or kFmtBF16); a_size / b_size: the operand buffers (doubles).
    int build(const GemmSchedule& s, int fmt, int64_t a_size, int64_t b_size, int64_t c_size, cudaStream_t st,
              int num_sms);
    // C (+)= the schedule's products: packs A and B, then one persistent launch.
    int run(const double* A, const double* B, double* C, bool accumulate, int* status, cudaStream_t st) const;
};

}  // namespace dmrg
