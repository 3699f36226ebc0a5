// Truncation bookkeeping (see truncate.h).
#include "truncate.h"

#include <utility>

namespace dmrg {

void quicksort_with_index(double* a, int* index, int n, bool descending) {
    std::vector<std::pair<int, int>> stack;
    stack.emplace_back(0, n - 1);
    while (!stack.empty()) {
        const int left = stack.back().first, right = stack.back().second;
        stack.pop_back();
        if (left >= right) continue;
        int i = left, j = right;
        const double pv = a[i];
        const int pi = index[i];
        if (descending) {
            while (i < j) {
                while (i < j && a[j] <= pv) --j;
                if (i < j) {
                    a[i] = a[j];
                    index[i] = index[j];
                    ++i;
                }
                while (i < j && a[i] >= pv) ++i;
                if (i < j) {
                    a[j] = a[i];
                    index[j] = index[i];
                    --j;
                }
            }
        } else {
            while (i < j) {
                while (i < j && a[j] >= pv) --j;
                if (i < j) {
                    a[i] = a[j];
                    index[i] = index[j];
                    ++i;
                }
                while (i < j && a[i] <= pv) ++i;
                if (i < j) {
                    a[j] = a[i];
                    index[j] = index[i];
                    --j;
                }
            }
        }
        a[i] = pv;
        index[i] = pi;
        stack.emplace_back(left, i - 1);
        stack.emplace_back(i + 1, right);
    }
}

std::vector<int> compute_truncate_dim(int max_dim, double canpre, std::vector<std::vector<double>>& svals) {
    if (canpre > 1) canpre = 0.0;
    const int ns = (int)svals.size();
    std::vector<int> t(ns, 0);
    int total = 0;
    for (int i = 0; i < ns; ++i) {
        for (double v : svals[i])
            if (v > canpre) ++t[i];
        total += t[i];
    }
    if (total > 0 && max_dim > 0 && max_dim < total) {
        std::vector<double> v;
        std::vector<int> blk;
        v.reserve(total);
        blk.reserve(total);
        for (int i = 0; i < ns; ++i)
            for (int j = 0; j < t[i]; ++j) {
                v.push_back(svals[i][j]);
                blk.push_back(i);
            }
        quicksort_with_index(v.data(), blk.data(), total, true);
        std::fill(t.begin(), t.end(), 0);
        for (int i = 0; i < max_dim; ++i) ++t[blk[i]];
    }
    for (int i = 0; i < ns; ++i)
        if (t[i] == 0) {
            t[i] = 1;
            if (!svals[i].empty()) svals[i][0] = 0.0;
        }
    return t;
}

double discarded_weight(const std::vector<std::vector<double>>& svals, const std::vector<int>& tdim) {
    double w = 0.0;
    for (size_t i = 0; i < svals.size(); ++i)
        for (size_t j = (size_t)tdim[i]; j < svals[i].size(); ++j) w += svals[i][j] * svals[i][j];
    return w;
}

}  // namespace dmrg
