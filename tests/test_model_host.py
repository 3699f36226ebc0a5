"""Model layer of the product library (host only): the MPO built by the
deparallelising term-by-term construction and the quantum-number tables are
bit-identical to the reference's (dumped by oracle/_ref/probe_dump)."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import build, capi
from oracle.nac import read_nac

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
CASES = [("chain16_spinless.in", "model_chain16.nac"), ("cylinder8x4_spinless.in", "model_cyl8x4.nac")]


@pytest.fixture(scope="module", autouse=True)
def _lib():
    try:
        build.nvcc()
        build.build()
    except RuntimeError:
        pass
    capi._lib = None
    capi.lib()


@pytest.mark.parametrize("inp,gold", CASES)
def test_mpo_and_quantum_tables_bit_exact(inp, gold):
    ref = read_nac(os.path.join(GOLD, gold))
    m = capi.Model(os.path.join(ROOT, "dmrgcc_b200", "inputs", inp))
    n = int(ref["num_site"][0])
    assert m.num_site == n
    for i in range(n):
        W = m.mpo(i)
        d, lb, rb = (int(x) for x in ref[f"op{i}.dims"])
        assert W.shape == (lb, rb, d, d)
        assert np.array_equal(W.ravel(), ref[f"op{i}.W"])  # bit-exact doubles
    for b in range(n + 1):
        assert np.array_equal(m.quantum_table(0, b).ravel(), ref[f"sq{b}"])
        assert np.array_equal(m.quantum_table(1, b).ravel(), ref[f"hq{b}"])
