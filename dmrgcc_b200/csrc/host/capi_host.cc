// C ABI entry points that only do host bookkeeping (callable without a GPU).
#include <vector>

#include "dmrg_b200.h"
#include "host/grand.h"
#include "truncate.h"

namespace dmrg {
int set_error(int code, const char* fmt, ...);
}

extern "C" {

int dmrg_rand_stream(unsigned seed, int n, int* out) {
    if (n < 0 || (n > 0 && !out)) return dmrg::set_error(DMRG_E_ARG, "invalid arguments");
    dmrg::GlibcRand rng(seed);
    for (int i = 0; i < n; ++i) out[i] = rng.next();
    return DMRG_OK;
}

int dmrg_quicksort_index(double* values, int* index, int n, int descending) {
    if (n < 0 || (n > 0 && (!values || !index))) return dmrg::set_error(DMRG_E_ARG, "invalid quicksort arguments");
    if (n > 0) dmrg::quicksort_with_index(values, index, n, descending != 0);
    return DMRG_OK;
}

int dmrg_truncate_dims(int nsec, const int* counts, double* values, int max_dim, double canpre, int* tdim_out) {
    if (nsec < 0 || (nsec > 0 && (!counts || !tdim_out))) return dmrg::set_error(DMRG_E_ARG, "invalid arguments");
    std::vector<std::vector<double>> s(nsec);
    int64_t pos = 0;
    for (int i = 0; i < nsec; ++i) {
        if (counts[i] < 0) return dmrg::set_error(DMRG_E_ARG, "negative count");
        s[i].assign(values + pos, values + pos + counts[i]);
        pos += counts[i];
    }
    std::vector<int> t = dmrg::compute_truncate_dim(max_dim, canpre, s);
    pos = 0;
    for (int i = 0; i < nsec; ++i) {
        tdim_out[i] = t[i];
        for (int j = 0; j < counts[i]; ++j) values[pos + j] = s[i][j];
        pos += counts[i];
    }
    return DMRG_OK;
}

}  // extern "C"
