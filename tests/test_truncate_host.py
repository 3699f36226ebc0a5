"""a7 bookkeeping in the product library (host code, CPU only): the library's
QuickSort and ComputeTruncateDim against the reference's own sort order
(golden cases from the reference's QuickSort) and the oracle."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import build, capi
from oracle import dmrg_oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module", autouse=True)
def _lib():
    try:
        build.nvcc()
        build.build()
    except RuntimeError:
        pass
    capi._lib = None
    capi.lib()


def test_library_quicksort_matches_reference_order():
    with open(os.path.join(GOLD, "quicksort_cases.txt")) as f:
        lines = f.read().strip().split("\n")
    for inp, out in zip(lines[0::2], lines[1::2]):
        toks = inp.split()
        n, flag = int(toks[0]), int(toks[1])
        vals = [float(x) for x in toks[2:2 + n]]
        _, idx = capi.quicksort_index(vals, descending=(flag == 0))
        assert list(idx) == [int(x) for x in out.split()]


@pytest.mark.parametrize("seed", range(20))
def test_library_truncation_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    nsec = int(rng.integers(1, 12))
    pool = np.array([1e-14, 1e-13, 1e-6, 0.01, 0.1, 0.25, 0.5])
    svals = [np.sort(rng.choice(pool, size=int(rng.integers(1, 9))))[::-1].copy() for _ in range(nsec)]
    max_dim = int(rng.integers(-1, 20))
    canpre = float(rng.choice([1e-12, 0.0, 2.0, 1e-7]))
    t_lib, s_lib = capi.truncate_dims([s.copy() for s in svals], max_dim, canpre)
    s_orc = [s.copy() for s in svals]
    t_orc = O.compute_truncate_dim(max_dim, canpre, s_orc)
    assert list(t_lib) == list(t_orc)
    for a, b in zip(s_lib, s_orc):
        assert np.array_equal(a, b)
