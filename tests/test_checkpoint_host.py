"""Checkpoint format (the on-disk tensor-space file), host side: the reader in
oracle/space_file.py restates the reference's writers; it must parse the file
the reference itself wrote (tests/golden/record_chain6.dat: the 6-site chain
after its first two sweeps, cache_record) completely and consistently with the
model's quantum tables and the sweep table."""
import os

import numpy as np

from dmrgcc_b200 import capi
from oracle.space_file import read_space

HERE = os.path.dirname(__file__)
GOLD = os.path.join(HERE, "golden")
INPUT = os.path.join(os.path.dirname(HERE), "dmrgcc_b200", "inputs", "chain6_spinless.in")


def test_reference_record_parses_and_matches_the_model():
    s = read_space(os.path.join(GOLD, "record_chain6.dat"))
    m = capi.Model(INPUT)
    try:
        assert s.num_site == m.num_site == 6 and s.num_quantum == m.num_quantum
        for b in range(s.num_site + 1):
            assert np.array_equal(s.quantum_table[b], m.quantum_table(0, b))
        for i, lat in enumerate(s.lattices):
            assert lat.physics_dim == m.physics_dim
            assert all(0 <= x < len(s.quantum_table[i]) for x in lat.left_block)
            assert all(0 <= x < len(s.quantum_table[i + 1]) for x in lat.right_block)
            assert lat.physics_index.shape == (len(lat.left_block), len(lat.right_block))
            for left, right, a in lat.blocks:
                assert lat.physics_index[left, right] >= 0
                assert np.all(np.isfinite(a))
    finally:
        m.close()
    # parameters of the last half-sweep before the record (4th row of the table)
    assert (s.max_block, s.max_dim, s.canonical_precision) == (100, 32, 1e-12)
    assert abs(s.noise_factor - 1e-5) <= 1e-20
