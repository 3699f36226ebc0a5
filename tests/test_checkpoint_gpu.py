"""Checkpoint write and resume (cache_record / cache_resume, the on-disk
tensor-space file) against the reference.

* Writing: the library's record of the 6-site chain after two sweeps equals the
  one the (sign-gauge-pinned) reference wrote for the same run
  (tests/golden/record_chain6.dat): same header, quantum tables, sectors, block
  lists and parameters, and the same state: the MPS of each file contracted
  into the full 3^6-component wavefunction, equal to 1e-9 (the site tensors
  themselves are fixed only up to rotations inside degenerate singular
  subspaces, so they are not compared element by element).
* Resuming: a run resumed from the reference's file follows the reference run
  resumed from it (tests/golden/trace_gauge_chain6_resume.txt; the reference's
  reader overruns its quantum-table arrays, so that run used a corrected reader
  with the same format, see oracle/probe/probe_dump.cc), by the alignment rule
  of tests/test_engine_gpu.py with energies to 1e-7 per site in the noisy
  half-sweeps (see the test), and to 1e-10 per site at the end.
* A truncated file or one of another model is refused with an error.
"""
import os
import re
import shutil

import numpy as np
import pytest

from dmrgcc_b200 import capi
from oracle.space_file import read_space
from test_engine_gpu import aligned_prefix, parse_trace

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(__file__)
GOLD = os.path.join(HERE, "golden")
INPUTS = os.path.join(os.path.dirname(HERE), "dmrgcc_b200", "inputs")
RECORD = os.path.join(GOLD, "record_chain6.dat")


def input_with(name, tmp_path, **values):
    src = open(os.path.join(INPUTS, f"{name}_spinless.in")).read()
    for k, v in values.items():
        src, n = re.subn(rf"(?m)^(\s*){k}\s*=.*$", rf"\g<1>{k} = {v}", src)
        assert n == 1, k
    path = str(tmp_path / f"{name}.in")
    with open(path, "w") as f:
        f.write(src)
    return path


def full_state(space):
    """The MPS of a checkpoint contracted into the dense wavefunction (physical
    indices site 0 first).  A bond's basis is the concatenation of the sectors
    of the site on its left, in that site's order; the site on its right finds
    each of its left sectors there by quantum-table row."""
    d = space.lattices[0].physics_dim
    psi = np.ones((1, 1))  # [physical states so far, bond]
    prev = {0: (0, 1)}     # quantum-table row of the bond -> (offset, dim)
    for lat in space.lattices:
        right, off = {}, 0
        for q, dim in zip(lat.right_block, lat.right_dim):
            right[q] = (off, dim)
            off += dim
        t = np.zeros((sum(v[1] for v in prev.values()), d, off))
        for l, r, a in lat.blocks:
            lo, ld = prev[lat.left_block[l]]
            ro, rd = right[lat.right_block[r]]
            assert a.shape == (ld, rd) == (lat.left_dim[l], lat.right_dim[r])
            t[lo:lo + ld, lat.physics_index[l, r], ro:ro + rd] = a
        psi = np.einsum("sa,apb->spb", psi, t).reshape(-1, off)
        prev = right
    return psi.reshape(-1)


def test_record_matches_reference_record(ctx, tmp_path):
    inp = input_with("chain6", tmp_path, num_sweep=2, cache_record="true", cache_name=str(tmp_path),
                     record_name="mine.dat")
    run = capi.Run(ctx, inp)
    run.execute()
    run.close()
    got, ref = read_space(str(tmp_path / "mine.dat")), read_space(RECORD)
    assert (got.num_site, got.num_quantum) == (ref.num_site, ref.num_quantum)
    for a, b in zip(got.quantum_table, ref.quantum_table):
        assert np.array_equal(a, b)
    assert (got.max_block, got.max_dim, got.canonical_precision, got.noise_factor) == \
        (ref.max_block, ref.max_dim, ref.canonical_precision, ref.noise_factor)
    for lg, lr in zip(got.lattices, ref.lattices):
        assert lg.physics_dim == lr.physics_dim
        assert (lg.left_block, lg.left_dim, lg.right_block, lg.right_dim) == \
            (lr.left_block, lr.left_dim, lr.right_block, lr.right_dim)
        assert np.array_equal(lg.physics_index, lr.physics_index)
        assert [(l, r, a.shape) for l, r, a in lg.blocks] == [(l, r, a.shape) for l, r, a in lr.blocks]
    psi_got, psi_ref = full_state(got), full_state(ref)
    assert abs(np.linalg.norm(psi_ref) - 1.0) <= 1e-10
    sign = 1.0 if float(psi_got @ psi_ref) >= 0 else -1.0
    assert np.max(np.abs(sign * psi_got - psi_ref)) <= 1e-9


def test_resume_from_reference_record_follows_reference(ctx, tmp_path):
    inp = input_with("chain6", tmp_path, cache_resume="true", resume_name=RECORD)
    trace = str(tmp_path / "trace.txt")
    os.environ["DMRG_TRACE"] = trace
    try:
        run = capi.Run(ctx, inp)
        run.execute()
    finally:
        del os.environ["DMRG_TRACE"]
    ref = parse_trace(os.path.join(GOLD, "trace_gauge_chain6_resume.txt"))
    got = parse_trace(trace)
    # The recorded state has degenerate singular values (the chain is mirror
    # symmetric), whose vectors are fixed only up to rotations; the subspace
    # expansion's random matrices act in that basis, so energies in the noisy
    # half-sweeps agree to ~1e-8 rather than to rounding.  Sector dimensions
    # must still agree operation by operation, and the final energies to 1e-10.
    n_aligned = aligned_prefix(ref, got, 1e-7 * 6)
    assert n_aligned >= min(len(ref), 250)
    rec = run.steps()
    stock = np.loadtxt(os.path.join(GOLD, "steps_chain6_resume.txt"))
    assert len(rec["energy"]) == len(stock)
    assert np.array_equal(rec["site"], stock[:, 1].astype(int))
    assert abs(rec["energy"][-1] - stock[-1, 4]) / 6 <= 1e-10
    run.close()


def test_resume_refuses_bad_files(ctx, tmp_path):
    cut = str(tmp_path / "cut.dat")
    with open(RECORD, "rb") as f:
        data = f.read()
    with open(cut, "wb") as f:
        f.write(data[: len(data) // 2])
    with pytest.raises(capi.DmrgError, match="truncated|malformed") as err:
        capi.Run(ctx, input_with("chain6", tmp_path, cache_resume="true", resume_name=cut))
    assert err.value.code == capi.E_IO
    other = input_with("chain16", tmp_path, cache_resume="true", resume_name=RECORD)
    with pytest.raises(capi.DmrgError, match="number of sites") as err:
        capi.Run(ctx, other)
    assert err.value.code == capi.E_IO
    missing = str(tmp_path / "none.dat")
    with pytest.raises(capi.DmrgError, match="cannot open") as err:
        capi.Run(ctx, input_with("chain6", tmp_path, cache_resume="true", resume_name=missing))
    assert err.value.code == capi.E_IO
