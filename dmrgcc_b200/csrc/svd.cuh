// Batched FP64 SVD of the sector matrices of one canonicalisation, on the device.
//
// Algorithm: one-sided (Hestenes) Jacobi with 32-column blocks.  Each sector
// matrix A (m x n) is held as a column-major working matrix W with c <= r
// columns: W = A when n <= m (right rotations accumulate V), W = A^T otherwise
// (they accumulate U).  A sweep first orders the columns by descending norm
// (de Rijk's pivoting, applied block-wise: blocks then hold columns of similar
// size, which halves the sweeps on noise-expanded tensors whose spectra are
// mostly tiny), then measures every pair of column blocks at once (the 32x32
// cross-Gram blocks of W, DMMA) and visits only the block pairs found
// unconverged, in as few rounds as a matching of them allows (the round-robin
// order restricted to them, or a greedy matching by measure if that needs
// fewer rounds).  In a round all pairs of all sectors are independent and each
// is split over CTAs by rows: (1) partial 64x64 Gram matrices of the pair over
// row ranges (DMMA), (2) one CTA per pair sums them and runs a few cyclic
// Jacobi sweeps on the Gram matrix in shared memory, (3) 64-row slices of the
// pair's columns of W and of the accumulated rotation are multiplied by the
// resulting 64x64 rotation (DMMA).  Converged when no pair has
// |g_ij| > tol ||A||_F max(|x_i|, |x_j|), tol = 2 eps sqrt(rows): the
// remaining non-orthogonality is a backward perturbation of A below rounding
// level, the accuracy of a backward-stable SVD such as the reference's dgesvd
// (singular values to ~eps ||A||, enough for its canpre cut at 1e-12 of a
// normalised state); columns of a rank-deficient matrix
// whose norm falls to rounding level (4 eps sqrt(rows) ||A||_F) are left out of
// rotations and of that test.  A matrix whose entries are all below 1/2 is
// first scaled by a power of two (exact) so that its largest entry lies in
// [0.5, 1), and scaled back at the end: the thresholds are relative, but their
// squared forms and the Gram entries of a sector with values near 1e-100 would
// underflow.  Singular values are the final column
// norms, sorted in descending order.  The free sign of each singular pair is
// fixed by a convention: the left singular vector's largest-magnitude component
// is positive (ties within a relative 1e-6: the first such component).
#pragma once

#include <vector>

#include "common.cuh"

namespace dmrg {

struct SvdProblem {
    int m, n;            // the sector matrix A is m x n
    int rows, cols;      // working matrix W: rows x cols, cols <= rows, column-major (ld = rows)
    int transposed;      // 1: W = A^T
    int nbe;             // number of 32-column blocks, rounded up to even (>= 2)
    int64_t w_off;       // offset of W in the W buffer (doubles)
    int64_t q_off;       // offset of the accumulated rotation (cols x cols, column-major)
    int64_t s_off;       // offset of the sorted singular values (cols doubles)
    int64_t perm_off;    // offset of the sort permutation (cols ints)
};

struct SvdTask {
    int problem;
    int bi, bj;            // the pair's column blocks (sorted order), bi < bj; bj may be an empty block
    int g_first, g_count;  // its Gram items, as indices into the round's item list
};

struct SvdTile {           // a 32x32 block of a sector's cross-Gram matrix (convergence measure)
    int problem;
    int bi, bj;            // bi <= bj
    int pad;
};


struct SvdItem {   // a row range of one pair task's columns
    int task;      // index into the task list
    int seg;       // 0: rows of W, 1: rows of the accumulated rotation
    int r0, r1;
};

class BatchedSvd {
public:
    // Plans the batch for the given sector shapes (m[i] x n[i]; entries with
    // m*n == 0 are skipped and report no singular values).
    int plan(const std::vector<int>& m, const std::vector<int>& n, cudaStream_t st);
    // Device address of sector i's working matrix W (fill it before run()).
    double* w(int i) const { return d_w.as<double>() + probs[index[i]].w_off; }
    bool active(int i) const { return index[i] >= 0; }
    const SvdProblem& problem(int i) const { return probs[index[i]]; }
    // Runs the Jacobi sweeps to convergence (sync per sweep) and sorts.
    int run(cudaStream_t st, int* sweeps_out = nullptr);
    // Sorted singular values of every active sector, copied to the host.
    int singular_values(std::vector<std::vector<double>>& out, cudaStream_t st);
    void dump_unconverged(const char* path, const DeviceBuffer& w_in, const std::vector<double>& worst,
                          cudaStream_t st);

    DeviceBuffer d_w, d_q, d_s, d_perm, d_probs, d_tasks, d_fro2;
    DeviceBuffer d_expo;  // per problem: the power of two W was scaled by (prescale_kernel)
    DeviceBuffer d_part;  // per problem and slice: largest magnitude, then sum of squares
    DeviceBuffer d_sign;  // +-1 per sorted singular triplet (sign convention, set by run())
    DeviceBuffer d_gram_items, d_rot_items, d_gpart, d_rot, d_skip;
    DeviceBuffer d_colmap, d_norm;  // per sweep: columns in descending norm order
    DeviceBuffer d_tiles, d_bm;     // the convergence measure's tiles and their values
    DeviceBuffer d_sched;           // lane order of the pair solve's rotations (uploaded once)
    std::vector<SvdProblem> probs;
    std::vector<int> index;             // sector -> problem (-1 when empty)
    std::vector<SvdTile> tiles;         // all block pairs bi <= bj of every problem
    std::vector<int> tile_first;        // per problem: its first tile
    int gram_rows = 64;                 // rows of a Gram item
    // the current sweep's rounds (rebuilt every sweep from the measure)
    std::vector<int> round_first;       // task offset of each round
    std::vector<SvdTask> tasks;
    std::vector<SvdItem> gram_items, rot_items;    // per round, contiguous
    std::vector<int> round_gram_first, round_rot_first;
    int max_tasks = 0, max_gram = 0, max_rot = 0;  // capacities (per sweep)
    int max_round_tasks = 0, max_round_gram = 0;   // capacities (per round)

private:
    // Builds the sweep's rounds from the block measures bm (tiles order);
    // returns the number of rounds (0: converged).
    int schedule(const std::vector<double>& bm);
    void add_task(int problem, int bi, int bj);
};

}  // namespace dmrg
