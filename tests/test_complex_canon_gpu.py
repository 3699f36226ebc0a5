"""Complex canonicalisation on the device (dmrg_zcanon_*: the batched Jacobi SVD
of each sector's real form, complex triplets recovered on the host) against the
reference's ComplexTensorLattice::Left/RightCanonicalTensorLattice (zgesdd) on
the subspace-expanded Hofstadter tensors of tests/golden/make_golden.py
--complex: truncation dimensions bit-exact; singular values (row / column norms
of S V^H / U S) within 1e-12; the gauge-invariant products U S V^H of every
block within 1e-11; the new ket orthonormal per sector."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from dmrgcc_b200.problem import read_nac

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _spec(d, p):
    return capi.BlockSpec(d[p + ".left"], d[p + ".right"], d[p + ".rows"], d[p + ".cols"])


def _blocks(flat, rows, cols):
    off = np.concatenate([[0], np.cumsum(np.asarray(rows, np.int64) * cols)])
    return [flat[off[k]:off[k + 1]].reshape(rows[k], cols[k]) for k in range(len(rows))]


@pytest.mark.parametrize("call", [244, 266])
def test_complex_canonical_matches_reference(ctx, call):
    d = read_nac(os.path.join(GOLD, f"zcanon_hof_c{call}.nac"))
    left = bool(d["left"][0])
    side = 0 if left else 1
    ket = _spec(d, "before.ket")
    c = capi.Canonical(ctx, side, d["before.left_dim"], d["before.right_dim"], ket, complex=True)
    kdev = capi.DeviceArray.from_host(ctx, np.asarray(d["before.ket.data"]))
    res = c.run(kdev, int(d["max_dim"][0]), float(d["canpre"][0]))
    assert np.array_equal(res["tdim"], d["after.right_dim"] if left else d["after.left_dim"])
    assert np.array_equal(res["ket_rows"], d["after.ket.rows"])
    assert np.array_equal(res["ket_cols"], d["after.ket.cols"])
    assert np.array_equal(res["canon_rows"], d["after.canonical.rows"])
    assert np.array_equal(res["canon_cols"], d["after.canonical.cols"])
    assert np.array_equal(res["match_dim"], d["after.match_dim"])
    newk = capi.DeviceArray(ctx, 2 * res["ket_size"])
    can = capi.DeviceArray(ctx, 2 * res["canonical_size"])
    c.write(kdev, newk, can)
    ctx.sync()
    kb = _blocks(newk.download().view(np.complex128), res["ket_rows"], res["ket_cols"])
    cb = _blocks(can.download().view(np.complex128), res["canon_rows"], res["canon_cols"])
    rkb = _blocks(np.asarray(d["after.ket.data"]).view(np.complex128), d["after.ket.rows"], d["after.ket.cols"])
    rcb = _blocks(np.asarray(d["after.canonical.data"]).view(np.complex128), d["after.canonical.rows"],
                  d["after.canonical.cols"])
    ax = 1 if left else 0
    for a, b in zip(cb, rcb):  # singular values
        assert np.allclose(np.linalg.norm(a, axis=ax), np.linalg.norm(b, axis=ax), rtol=0, atol=1e-12)
    sec = d["after.ket.right"] if left else d["after.ket.left"]
    for k in range(len(kb)):  # gauge-invariant products
        s = sec[k]
        mine = kb[k] @ cb[s] if left else cb[s] @ kb[k]
        ref = rkb[k] @ rcb[s] if left else rcb[s] @ rkb[k]
        assert np.allclose(mine, ref, atol=1e-11)
    nsec = len(res["tdim"])
    for s in range(nsec):  # orthonormal new ket per sector
        mem = [k for k in range(len(kb)) if sec[k] == s]
        if not mem or res["tdim"][s] == 0:
            continue
        M = np.vstack([kb[k] for k in mem]) if left else np.hstack([kb[k] for k in mem])
        G = M.conj().T @ M if left else M @ M.conj().T
        if np.linalg.norm(cb[s]) > 0:
            assert np.allclose(G, np.eye(G.shape[0]), atol=1e-10)
