"""Pins the numpy oracle to the reference at bond dimension 1024 (8x4 cylinder),
on the compact fixtures of tests/golden/make_golden.py --d1024: the block
structures the reference had at that point of its run, the seeded synthetic
inputs it then computed on (regenerated here from the seed) and digests of its
outputs.  This also checks the fixture pipeline that the GPU tests
(test_d1024_gpu.py) rely on.  CPU only; a few seconds per case."""
import os

import numpy as np
import pytest

from oracle import dmrg_oracle as O
from oracle.nac import read_nac

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _fill(blist, values, pos):
    for k, m in enumerate(blist.mats):
        n = m.size
        blist.mats[k] = values[pos:pos + n].reshape(m.shape).copy()
        pos += n
    return pos


def _case(path):
    if not os.path.exists(path):
        pytest.skip(f"{os.path.basename(path)} not generated")
    return read_nac(path)


@pytest.mark.parametrize("call", [283, 314])
def test_oracle_env_update_D1024(call):
    d = _case(os.path.join(GOLD, f"env_cyl8x4_D1024_c{call}.nac"))
    lat, W = O.lattice_from_nac(d, "lattice"), O.operator_from_nac(d, "op")
    env_in = O.env_from_nac(d, "env_in")
    n = lat.psi_dim() + sum(m.size for e in env_in for m in e.mats)
    vals = O.splitmix_uniform(int(d["synth_seed"][0]), 0, n)
    pos = _fill(lat.ket, vals, 0)
    for e in env_in:
        pos = _fill(e, vals, pos)
    fn = O.left_compute_env if d["left"][0] else O.right_compute_env
    out = fn(lat, W, env_in)
    ref_struct = O.env_from_nac(d, "env_out")
    assert len(out) == len(ref_struct)
    for a, b in zip(out, ref_struct):
        assert a.left == b.left and a.right == b.right
        assert [m.shape for m in a.mats] == [m.shape for m in b.mats]
    flat = np.concatenate([m.ravel() for e in out for m in e.mats])
    ref = np.asarray(d["digest.value"])
    assert np.max(np.abs(flat[d["digest.index"]] - ref)) <= 1e-13 * np.max(np.abs(ref))
    sumsq = [sum(float(np.sum(m * m)) for m in e.mats) for e in out]
    assert np.allclose(sumsq, d["digest.sumsq"], rtol=1e-12)


@pytest.mark.parametrize("call", [318, 349])
def test_oracle_canonical_D1024(call):
    d = _case(os.path.join(GOLD, f"canon_cyl8x4_D1024_c{call}.nac"))
    lat = O.lattice_from_nac(d, "before")
    after = O.lattice_from_nac(d, "after")
    left = bool(d["left"][0])
    _fill(lat.ket, O.splitmix_uniform(int(d["synth_seed"][0]), 0, lat.psi_dim()), 0)
    fn = O.left_canonical if left else O.right_canonical
    fn(lat, int(d["max_dim"][0]), float(d["canpre"][0]))
    assert lat.left_dim == after.left_dim and lat.right_dim == after.right_dim
    assert [m.shape for m in lat.ket.mats] == [m.shape for m in after.ket.mats]
    assert lat.match_dim == after.match_dim
    ax = 1 if left else 0
    sig = np.concatenate([np.linalg.norm(m, axis=ax) for m in lat.canonical.mats])
    assert np.allclose(np.sort(sig), np.sort(np.asarray(d["digest.sigma"])), rtol=0,
                       atol=1e-12 * float(np.max(d["digest.sigma"])))
    prods = []
    for k, b in enumerate(lat.ket.mats):
        s = lat.ket.right[k] if left else lat.ket.left[k]
        c = lat.canonical.mats[s]
        prods.append((b @ c if left else c @ b).ravel())
    flat = np.concatenate(prods)
    ref = np.asarray(d["digest.value"])
    assert np.max(np.abs(flat[d["digest.index"]] - ref)) <= 1e-11 * np.max(np.abs(ref))


def test_oracle_lanczos_D1024():
    path = os.path.join(GOLD, "lanczos_cyl8x4_D1024_c252.npz")
    if not os.path.exists(path):
        pytest.skip("lanczos_cyl8x4_D1024_c252.npz not generated")
    z = np.load(path)
    d = {k: z[k] for k in z.files}
    for k in list(d):
        if d[k].dtype == np.float32:
            d[k] = d[k].astype(np.float64)
    lat, W = O.lattice_from_nac(d, "lattice"), O.operator_from_nac(d, "op")
    L, R = O.env_from_nac(d, "L"), O.env_from_nac(d, "R")
    res = O.lanczos(lat, W, L, R, int(d["niter"][0]))
    assert abs(res["energy"] - float(d["energy"][0])) / 32 <= 1e-12
    g = d["ground"] / np.linalg.norm(d["ground"])
    assert 1.0 - abs(float(lat.ket.vectorize() @ g)) <= 1e-7
