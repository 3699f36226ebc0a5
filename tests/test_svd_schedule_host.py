"""The batched SVD's pair-solve schedule (svd.cu, build_pair_schedule), checked
independently of the library's own checks: each of the 63 steps rotates 32
disjoint column pairs covering all 64 columns, every two columns share exactly
one step (a cyclic sweep of the pair's Gram matrix, as the round-robin order it
reorders), and in each half-warp the 16 columns addressed first, and the 16
addressed second, are distinct mod 16 (8-byte shared-memory banks)."""
import numpy as np

from dmrgcc_b200 import capi


def test_pair_schedule_is_a_cyclic_sweep_without_bank_collisions():
    tab = capi.svd_pair_schedule().astype(np.int64)
    a, b, flip = tab & 63, (tab >> 6) & 63, (tab >> 12) & 1
    assert np.all(a < b) and np.all(tab >> 13 == 0)
    met = np.zeros((64, 64), dtype=np.int64)
    for r in range(63):
        assert sorted(np.concatenate([a[r], b[r]]).tolist()) == list(range(64))
        np.add.at(met, (a[r], b[r]), 1)
        first = np.where(flip[r] == 1, b[r], a[r])
        second = np.where(flip[r] == 1, a[r], b[r])
        for h in (slice(0, 16), slice(16, 32)):
            assert len(set((first[h] % 16).tolist())) == 16
            assert len(set((second[h] % 16).tolist())) == 16
    assert np.array_equal(met[np.triu_indices(64, 1)], np.ones(64 * 63 // 2, dtype=np.int64))
