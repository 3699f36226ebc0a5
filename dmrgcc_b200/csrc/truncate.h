// a7: truncation rule of the reference, on the host (integer bookkeeping must be
// bit-exact, including the tie order of its unstable quicksort).
#pragma once

#include <vector>

namespace dmrg {

// In-place quicksort with a companion index array; first element as pivot,
// descending when `descending`, else ascending.  Same partition steps as the
// reference's QuickSort(T*, int*, left, right, flag) (src/util/general.ih:7-65),
// so ties end up in the same order.  Sub-ranges are processed through an
// explicit stack (their order does not change the result: they are disjoint).
void quicksort_with_index(double* a, int* index, int n, bool descending);

// RealTensorLattice::ComputeTruncateDim (src/dmrg/realdmrg/real_tensor_lattice.cc:501-555):
// per sector, count singular values > canpre (canpre > 1 means 0); if the total
// exceeds max_dim > 0, keep the max_dim largest overall (global sort); a sector
// left with none keeps one value forced to 0.  `svals` is modified like the
// reference modifies its array.
std::vector<int> compute_truncate_dim(int max_dim, double canpre, std::vector<std::vector<double>>& svals);

// Sum of the squares of the singular values that were not kept (from the
// unmodified values).
double discarded_weight(const std::vector<std::vector<double>>& svals, const std::vector<int>& tdim);

}  // namespace dmrg
