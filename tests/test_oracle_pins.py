"""Pins the numpy oracle (oracle/dmrg_oracle.py) to the reference itself.

The fixtures under tests/golden/ were produced by the unmodified reference built
from its sources (oracle/Makefile) and instrumented by oracle/probe/probe_dump.cc
(tests/golden/make_golden.py).  CPU only."""
import os

import numpy as np
import pytest

from oracle import dmrg_oracle as O
from oracle.nac import read_nac

GOLD = os.path.join(os.path.dirname(__file__), "golden")
HEFF = ["heff_c20.nac", "heff_c158.nac"]


def _load_heff(name):
    d = read_nac(os.path.join(GOLD, name))
    return d, O.lattice_from_nac(d, "lattice"), O.operator_from_nac(d, "op"), O.env_from_nac(d, "L"), \
        O.env_from_nac(d, "R")


@pytest.mark.parametrize("name", HEFF)
def test_heff_matches_reference(name):
    d, lat, W, L, R = _load_heff(name)
    out = np.zeros(lat.psi_dim())
    O.multiply_effect_hamilton(lat, W, L, R, out)
    ref = d["heff_out"]
    assert np.max(np.abs(out - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_dense_heff_matches_reference():
    d, lat, W, L, R = _load_heff("heff_c20.nac")
    H = O.compute_effect_hamilton(lat, W, L, R)
    assert np.max(np.abs(H.ravel() - d["heff_dense"])) <= 1e-13 * np.max(np.abs(H))
    # H_eff is symmetric and agrees with the matvec
    assert np.allclose(H, H.T, atol=1e-12)
    psi = lat.ket.vectorize()
    out = np.zeros_like(psi)
    O.multiply_effect_hamilton(lat, W, L, R, out)
    assert np.allclose(H @ psi, out, atol=1e-12)


@pytest.mark.parametrize("call", [20, 158])
def test_lanczos_matches_reference(call):
    d, lat, W, L, R = _load_heff(f"heff_c{call}.nac")
    ref = read_nac(os.path.join(GOLD, f"lanczos_c{call}.nac"))
    res = O.lanczos(lat, W, L, R, int(d["niter"][0]))
    n_sites = 16
    assert abs(res["energy"] - ref["energy"][0]) / n_sites <= 1e-12
    v_ref = O.lattice_from_nac(ref, "lattice").ket.vectorize()
    assert abs(abs(lat.ket.vectorize() @ v_ref) - 1.0) <= 1e-10


@pytest.mark.parametrize("call", [173, 187])
def test_env_update_matches_reference(call):
    d = read_nac(os.path.join(GOLD, f"env_c{call}.nac"))
    lat, W = O.lattice_from_nac(d, "lattice"), O.operator_from_nac(d, "op")
    env_in, env_out = O.env_from_nac(d, "env_in"), O.env_from_nac(d, "env_out")
    fn = O.left_compute_env if d["left"][0] else O.right_compute_env
    out = fn(lat, W, env_in)
    assert len(out) == len(env_out)
    scale = max(np.max(np.abs(m)) for e in env_out for m in e.mats if m.size)
    for a, b in zip(out, env_out):
        assert a.left == b.left and a.right == b.right  # block maps bit-exact
        for x, y in zip(a.mats, b.mats):
            assert x.shape == y.shape
            assert np.max(np.abs(x - y), initial=0.0) <= 1e-13 * scale


@pytest.mark.parametrize("call", [160, 174])
def test_canonical_matches_reference(call):
    d = read_nac(os.path.join(GOLD, f"canon_c{call}.nac"))
    lat, after = O.lattice_from_nac(d, "before"), O.lattice_from_nac(d, "after")
    left = bool(d["left"][0])
    before = O.lattice_from_nac(d, "before")
    fn = O.left_canonical if left else O.right_canonical
    info = fn(lat, int(d["max_dim"][0]), float(d["canpre"][0]))
    # truncation dimensions: bit-exact
    assert lat.left_dim == after.left_dim and lat.right_dim == after.right_dim
    assert [m.shape for m in lat.ket.mats] == [m.shape for m in after.ket.mats]
    assert lat.match_dim == after.match_dim
    # singular values (row/column norms of S V^T or U S) agree
    for a, b in zip(lat.canonical.mats, after.canonical.mats):
        ax = 1 if left else 0
        assert np.allclose(np.linalg.norm(a, axis=ax), np.linalg.norm(b, axis=ax), rtol=0, atol=1e-12)
    # gauge-invariant: the kept product ket * canonical reproduces the reference's
    nsec = len(lat.canonical.mats)
    for s in range(nsec):
        pos = lat.ket.same_index(1 if left else 0, s)
        for p in pos:
            if left:
                mine = lat.ket.mats[p] @ lat.canonical.mats[s]
                ref = after.ket.mats[p] @ after.canonical.mats[s]
            else:
                mine = lat.canonical.mats[s] @ lat.ket.mats[p]
                ref = after.canonical.mats[s] @ after.ket.mats[p]
            assert np.allclose(mine, ref, atol=1e-11)
    assert info["discarded"] >= 0.0
    assert before.psi_dim() >= lat.psi_dim()


def test_quicksort_port_tie_breaking():
    # Arrays with many equal keys: the port must reproduce the index order of the
    # reference's unstable QuickSort (src/util/general.ih:7-65) exactly.
    with open(os.path.join(GOLD, "quicksort_cases.txt")) as f:
        lines = f.read().strip().split("\n")
    assert len(lines) == 80
    for inp, out in zip(lines[0::2], lines[1::2]):
        toks = inp.split()
        n, flag = int(toks[0]), int(toks[1])
        vals = [float(x) for x in toks[2:2 + n]]
        idx = list(range(n))
        O.quicksort_with_index(vals, idx, descending=(flag == 0))
        assert idx == [int(x) for x in out.split()]


def test_truncate_dim_rules():
    # canpre filter, global max_dim cut, empty sector forced to one zero value
    s = [np.array([0.9, 0.3, 1e-13]), np.array([0.5, 0.4]), np.array([1e-14])]
    t = O.compute_truncate_dim(3, 1e-12, s)
    assert t == [1, 2, 1] and s[2][0] == 0.0
    s = [np.array([0.9, 0.3]), np.array([0.5])]
    assert O.compute_truncate_dim(-1, 0.0, s) == [2, 1]
    # canpre > 1 is treated as 0
    assert O.compute_truncate_dim(10, 2.0, [np.array([0.1, 0.0])]) == [1]


def test_reference_energy_trajectory_monotone_at_end():
    rows = np.loadtxt(os.path.join(GOLD, "steps_chain16.txt"))
    assert rows.shape[1] == 6 and len(rows) == 180
    final = rows[-1, 4]
    assert abs(final - (-13.539043419078)) < 1e-9


@pytest.mark.parametrize("call", [38, 50])
def test_merge_matches_reference(call):
    """a8: the oracle's Left/RightMergeTensorLattice + NormalizeTensorLattice
    against the reference's own merge on the 16-site chain (merge call 38: left,
    50: right; site 9 of the second sweep): sector dimensions and block shapes
    exact, values to 1e-13 of the largest (the reference's products are
    OpenBLAS dgemm calls, the oracle's numpy's)."""
    d = read_nac(os.path.join(GOLD, f"merge_c{call}.nac"))
    side = int(d["side"][0])
    before = O.lattice_from_nac(d, "before")
    source = O.lattice_from_nac(d, "source")
    after = O.lattice_from_nac(d, "after")
    got = O.merge_lattice(before, source, side)
    assert got.left_dim == after.left_dim and got.right_dim == after.right_dim
    assert got.ket.left == after.ket.left and got.ket.right == after.ket.right
    scale = max(float(np.max(np.abs(m))) for m in after.ket.mats if m.size)
    for g, w in zip(got.ket.mats, after.ket.mats):
        assert g.shape == w.shape
        if w.size:
            assert np.max(np.abs(g - w)) <= 1e-13 * scale
    # the merge changes the merged side's dimensions where the truncation did
    changed = (before.left_dim != after.left_dim) if side == 0 else (before.right_dim != after.right_dim)
    assert changed
    assert abs(sum(float(np.sum(m * m)) for m in got.ket.mats) - 1.0) < 1e-13
