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

    // Copies the groups and terms of another schedule (not its execution form).
    void copy_plan(const GemmSchedule& o) {
        reset();
        terms = o.terms;
        groups = o.groups;
        ta = o.ta;
        tb = o.tb;
        flops = o.flops;
    }
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

// The same on the tcgen05 tensor cores with TF32 hi/lo splits (gemm_tf32x3.cu);
// `s` must be finalized with 128 x 64 x 32 tiles.  A wait that times out sets
// *status = DMRG_E_NUMERIC (device word) instead of hanging.
int launch_gemm_tf32x3(const GemmSchedule& s, const double* A, const double* B, double* C, bool accumulate,
                       int* status, cudaStream_t stream);

}  // namespace dmrg
