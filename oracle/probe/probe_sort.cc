// Test infrastructure: runs the reference's QuickSort with index
// (src/util/general.ih:7-65) on arrays read from stdin and prints the result,
// to pin the oracle's port of its tie-breaking.
// Input: repeated "n flag v_0 ... v_{n-1}" (flag 0 = descending, 1 = ascending).
// Output per case: the sorted values' original indices, one line.
#include "probe_common.h"

int main() {
    int n, flag;
    while (std::scanf("%d %d", &n, &flag) == 2) {
        std::vector<double> v(n);
        std::vector<int> idx(n);
        for (int i = 0; i < n; ++i) {
            if (std::scanf("%lf", &v[i]) != 1) return 1;
            idx[i] = i;
        }
        if (n > 0) QuickSort<double>(v.data(), idx.data(), 0, n - 1, flag);
        for (int i = 0; i < n; ++i) std::printf("%d%c", idx[i], i + 1 < n ? ' ' : '\n');
        if (n == 0) std::printf("\n");
    }
    return 0;
}
