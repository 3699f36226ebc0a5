"""The engine's random source against glibc itself: the reference draws its
initial MPS and its expansion matrices from srand/rand, and every block
structure of a run depends on those numbers.  The engine keeps its own copy of
the generator (no process-wide state, no lock); it must give the same stream."""
import ctypes

import numpy as np
import pytest

from dmrgcc_b200 import capi


@pytest.mark.parametrize("seed", [1, 2, 7, 12345, 2**31 - 1])
def test_rand_stream_equals_glibc(seed):
    libc = ctypes.CDLL(None)
    libc.srand(ctypes.c_uint(seed))
    want = np.array([libc.rand() for _ in range(5000)], dtype=np.int32)
    got = np.zeros(5000, dtype=np.int32)
    capi.check(capi.lib().dmrg_rand_stream(seed, 5000, got.ctypes.data_as(ctypes.POINTER(ctypes.c_int))),
               "dmrg_rand_stream")
    assert np.array_equal(got, want)
