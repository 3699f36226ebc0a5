// Two-site DMRG on the block-sparse engine: the split of the two-site tensor
// Theta into the two site tensors by a per-middle-sector SVD.
//
// Theta(k, p1, p2, l) has one block per (left sector k, middle sector c, right
// sector l) with p1 = p(k, c) and p2 = p(c, l) both allowed; the blocks of one
// middle sector c form the dense matrix M_c whose row blocks are its left
// sectors (a(k) rows each) and whose column blocks are its right sectors
// (b(l) columns each).  M_c = U S V^T per sector (BatchedSvd, one batch), a
// global truncation keeps the largest singular values, and
//   left to right:  K_j(k, c) = U rows of k,        K_{j+1}(c, l) = S V^T columns of l
//   right to left:  K_j(k, c) = U S rows of k,      K_{j+1}(c, l) = V^T columns of l.
// The reference has no two-site mode (its sweep is single-site with subspace
// expansion, real_tensor_rundmrg.cc:145-214); this is the engine's own.
// The factor that stays canonical (U left to right, V^T right to left) is
// orthonormal to rounding: where the Jacobi SVD leaves it as normalised
// working-matrix columns it is orthonormalised (KetOrtho) and the other factor
// is the projection of M_c on it (K^T M_c, or M_c K).
#pragma once

#include <vector>

#include "svd.cuh"

namespace dmrg {

struct SplitBlock {   // a Theta block and its place in its sector matrix
    int64_t theta_off;
    int rows, cols;
    int sector;       // index into the batch (candidate middle sector)
    int row0, col0;
};

struct SplitWrite {   // a block of a new site tensor
    int64_t out_off;
    int rows, cols;
    int sector;
    int off;          // part 0: first row of the block in M_c; part 1: first column
    int part;         // 0: left factor (rows of U), 1: right factor (columns of V^T)
    int64_t k_off;    // >= 0: the canonical factor's orthonormalised columns (column-major, ld = W rows)
    int64_t p_off;    // >= 0: the other factor as a projection, row-major (t x n_c, or m_c x t)
};

// Fills the batch's working matrices from Theta (zeroing them first); with
// `dst`, a buffer of the same layout instead.
int twosite_gather(BatchedSvd& svd, const std::vector<int>& sector_batch, const double* theta,
                   const std::vector<SplitBlock>& blocks, DeviceBuffer& d_blocks, cudaStream_t st,
                   double* dst = nullptr);

// Writes the new site tensors: left factor blocks into `left`, right factor
// blocks into `right`; `s_left` puts the singular values into the left factor
// (right-to-left sweep) instead of the right one.
// K: the orthonormalised columns (writes with k_off >= 0), P: the projected
// factors (writes with p_off >= 0).
int twosite_write(BatchedSvd& svd, const std::vector<int>& sector_batch, const std::vector<SplitWrite>& writes,
                  DeviceBuffer& d_writes, double* left, double* right, bool s_left, cudaStream_t st,
                  const double* K = nullptr, const double* P = nullptr);

// Global truncation of the two-site split: every singular value above canpre
// (canpre > 1: none), and of those the max_dim largest when max_dim > 0
// (descending, ties by sector then position).  A sector may keep nothing.
std::vector<int> truncate_twosite(int max_dim, double canpre, const std::vector<std::vector<double>>& svals);

}  // namespace dmrg
