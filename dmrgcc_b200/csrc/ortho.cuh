// Orthonormal kept columns from the batched Jacobi SVD.
//
// A sector's singular vectors on the side the Jacobi sweeps accumulate (V when
// W = A, U when W = A^T) are orthonormal to FP64 rounding.  Those on the other
// side are the working matrix's columns divided by their norms, and the sweeps'
// convergence test (a backward error of eps ||A||) leaves two such vectors of
// values s_i, s_j non-orthogonal by up to tol ||A||_F / min(s_i, s_j): ~1e-2 for
// values near 1e-12 of a normalised state.  Where a caller's new site tensor
// takes that side, KetOrtho forms the kept columns K0 (sign_j W[:, perm_j] / s_j)
// and orthonormalises them in descending order: K <- K (I - strictly upper part
// of K^T K), columns renormalised, each pass squaring the departure from
// orthonormality, as many passes as take the sector's bound below 1e-16 (plus
// one).  K = K0 R with R upper triangular near the identity (Gram-Schmidt in
// effect), so the large-s columns are left as they were, and the caller forms
// the other factor as the projection of the sector matrix on K (K^T A or A K):
// that equals diag(S) V^T (or U diag(S)) to eps ||A||.
#pragma once

#include <vector>

#include "gemm.cuh"
#include "svd.cuh"

namespace dmrg {

struct OrthoTask {
    int problem;     // batch problem
    int t, r;        // kept columns; rows of the working matrix
    int pad_;
    int64_t k_off;   // its columns in the K buffers (column-major, ld r)
    int64_t g_off;   // its t x t Gram matrix (row-major)
};

class KetOrtho {
public:
    // kept[i]: columns to orthonormalise for batch problem i (0: none).  The
    // number of passes follows each problem's bound tol ||A||_F / s_t from its
    // singular values (the batch's, as sorted by BatchedSvd::run).
    int plan(const BatchedSvd& svd, const std::vector<int>& kept, const std::vector<std::vector<double>>& sv,
             cudaStream_t st, int num_sms);
    // K0 from the batch's working matrix, then the passes.
    int run(const BatchedSvd& svd, cudaStream_t st);
    bool empty() const { return tasks.empty(); }
    // the orthonormalised columns after run(); k_off(problem) < 0: none
    const double* k() const { return (passes % 2 == 0 ? d_k : d_k2).as<double>(); }
    int64_t k_off(int problem) const {
        return problem >= 0 && problem < (int)koff.size() ? koff[problem] : -1;
    }
    int64_t k_size() const { return ksize; }
    const std::vector<OrthoTask>& task_list() const { return tasks; }

private:
    std::vector<OrthoTask> tasks;
    std::vector<int64_t> koff;  // by batch problem
    int64_t ksize = 0, gsize = 0;
    int cols = 0, passes = 0;
    DeviceBuffer d_tasks, d_k, d_k2, d_g;
    GemmSchedule sg, su;        // K^T K; K2 -= L K (L: the strictly lower part of K^T K)
};

}  // namespace dmrg
