// Grouped multi-term complex block GEMM (complex128, interleaved re/im like the
// reference's Complex, src/tensor/complex.h:11-76, and cuDoubleComplex): the
// contraction engine of the complex path (ComplexMatrix::MultiplyToMatrix ->
// cblas_zgemm, src/tensor/complex_matrix.cc:294-318).
//
// Same shape as the real engine (gemm.cuh): a launch processes output blocks
// ("groups"), each summing its terms  s_t * op(A_t) @ op(B_t)  in registers, with
// a complex scale s_t; op() may transpose (schedule-wide TA / TB) and conjugate
// (per term: bit 0 conjugates A, bit 1 conjugates B).  Offsets and leading
// dimensions count complex elements.
#pragma once

#include <cstdint>
#include <vector>

#include "common.cuh"
#include "gemm.cuh"

namespace dmrg {

struct ZGemmTerm {
    int64_t a_off;
    int64_t b_off;
    int lda;
    int ldb;
    int k;
    int conj;  // bit 0: conj(A), bit 1: conj(B)
    double s_re, s_im;
};

struct ZGemmSchedule {
    std::vector<ZGemmTerm> terms;
    std::vector<GemmGroup> groups;  // GemmGroup::cbuf unused (no split-K)
    std::vector<GemmTile> tiles;
    bool ta = false, tb = false;
    double flops = 0.0;  // real FLOPs: 8 m n k per term
    DeviceBuffer d_terms, d_groups, d_tiles;

    void reset() {
        terms.clear();
        groups.clear();
        tiles.clear();
        ta = tb = false;
        flops = 0.0;
    }
    int add_group(int64_t c_off, int ldc, int m, int n) {
        groups.push_back(GemmGroup{c_off, ldc, m, n, (int)terms.size(), (int)terms.size(), 0});
        return (int)groups.size() - 1;
    }
    void add_term(int64_t a_off, int lda, int64_t b_off, int ldb, int k, double s_re, double s_im, int conj = 0) {
        GemmGroup& g = groups.back();
        terms.push_back(ZGemmTerm{a_off, b_off, lda, ldb, k, conj, s_re, s_im});
        g.t1 = (int)terms.size();
        flops += 8.0 * g.m * g.n * (double)k;
    }
    // Every read of A/B and write of C inside buffers of the given sizes
    // (complex elements); DMRG_E_ARG otherwise.
    int check_bounds(int64_t a_size, int64_t b_size, int64_t c_size) const;
    // Tiles (64 x 32 complex, heaviest first) and upload.
    int finalize(cudaStream_t stream);
};

// C (+)= sum of terms for every tile of `s` (A, B, C: interleaved complex).
int launch_zgemm(const ZGemmSchedule& s, const double* A, const double* B, double* C, bool accumulate,
                 cudaStream_t stream);

}  // namespace dmrg
