"""a6/a7 parity: device SVD canonicalisation against the reference's
LeftCanonicalTensorLattice / RightCanonicalTensorLattice outputs.
Truncation dimensions bit-exact; singular values within 1e-12 absolute; the
gauge-invariant products (ket * canonical) within 1e-11; the new ket blocks
orthonormal per sector within 1e-12."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from dmrgcc_b200.problem import read_nac

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _blocks(d, p):
    return [np.asarray(d[p + k]) for k in (".left", ".right", ".rows", ".cols")]


@pytest.mark.parametrize("call", [160, 174])
def test_canonical_matches_reference(ctx, call):
    d = read_nac(os.path.join(GOLD, f"canon_c{call}.nac"))
    side = 0 if d["left"][0] else 1
    l, r, rows, cols = _blocks(d, "before.ket")
    ket = capi.BlockSpec(l, r, rows, cols)
    c = capi.Canonical(ctx, side, d["before.left_dim"], d["before.right_dim"], ket)
    kdev = capi.DeviceArray.from_host(ctx, d["before.ket.data"])
    res = c.run(kdev, int(d["max_dim"][0]), float(d["canpre"][0]))
    # bookkeeping: dims identical to the reference
    ref_dims = d["after.right_dim"] if side == 0 else d["after.left_dim"]
    assert np.array_equal(res["tdim"], ref_dims)
    ar, ac = _blocks(d, "after.ket")[2:]
    assert np.array_equal(res["ket_rows"], ar) and np.array_equal(res["ket_cols"], ac)
    cr, cc = _blocks(d, "after.canonical")[2:]
    assert np.array_equal(res["canon_rows"], cr) and np.array_equal(res["canon_cols"], cc)
    assert np.array_equal(res["match_dim"], d["after.match_dim"])
    newk = capi.DeviceArray(ctx, res["ket_size"])
    can = capi.DeviceArray(ctx, res["canonical_size"])
    c.write(kdev, newk, can)
    ctx.sync()
    K = newk.download()
    Cn = can.download()
    Kref = np.asarray(d["after.ket.data"])
    Cref = np.asarray(d["after.canonical.data"])

    def split(flat, rr, cc_):
        out, pos = [], 0
        for a, b in zip(rr, cc_):
            out.append(flat[pos:pos + a * b].reshape(a, b))
            pos += a * b
        return out

    kb, kbr = split(K, ar, ac), split(Kref, ar, ac)
    cb, cbr = split(Cn, cr, cc), split(Cref, cr, cc)
    nsec = len(cb)
    for s in range(nsec):
        # singular values = row (left) / column (right) norms of the canonical block
        ax = 1 if side == 0 else 0
        assert np.allclose(np.linalg.norm(cb[s], axis=ax), np.linalg.norm(cbr[s], axis=ax), rtol=0, atol=1e-12)
        members = [p for p in range(len(l)) if (r[p] if side == 0 else l[p]) == s]
        # orthonormality of the new blocks within the sector
        if members and min(kb[p].size for p in members) > 0:
            stack = np.vstack([kb[p] for p in members]) if side == 0 else np.hstack([kb[p] for p in members])
            gram = stack.T @ stack if side == 0 else stack @ stack.T
            if np.linalg.norm(cb[s]) > 0:
                assert np.allclose(gram, np.eye(gram.shape[0]), atol=1e-12)
        for p in members:
            mine = kb[p] @ cb[s] if side == 0 else cb[s] @ kb[p]
            ref = kbr[p] @ cbr[s] if side == 0 else cbr[s] @ kbr[p]
            assert np.allclose(mine, ref, atol=1e-11)
    assert res["discarded"] >= 0.0


def test_svd_sweep_cap_returns_numeric_error(ctx):
    """Fault injection on the host: with the Jacobi sweep cap lowered to one
    sweep, the canonicalisation of a D=64 tensor cannot converge and returns
    DMRG_E_NUMERIC with a message (the reference exits on a failed dgesvd,
    src/tensor/real_matrix.cc:615-619); with the cap restored the same call
    succeeds on the same context.  No device fault is involved: the cap is the
    host loop's."""
    d = read_nac(os.path.join(GOLD, "canon_c160.nac"))
    l, r, rows, cols = _blocks(d, "before.ket")
    ket = capi.BlockSpec(l, r, rows, cols)
    kdev = capi.DeviceArray.from_host(ctx, d["before.ket.data"])
    lib = capi.lib()
    try:
        assert lib.dmrg_svd_set_max_sweeps(1) == 0
        c = capi.Canonical(ctx, 0, d["before.left_dim"], d["before.right_dim"], ket)
        with pytest.raises(capi.DmrgError) as err:
            c.run(kdev, int(d["max_dim"][0]), float(d["canpre"][0]))
        assert err.value.code == capi.E_NUMERIC
        assert "did not converge" in str(err.value)
    finally:
        lib.dmrg_svd_set_max_sweeps(0)
    c = capi.Canonical(ctx, 0, d["before.left_dim"], d["before.right_dim"], ket)
    res = c.run(kdev, int(d["max_dim"][0]), float(d["canpre"][0]))
    assert np.array_equal(res["tdim"], d["after.right_dim"])


@pytest.mark.parametrize("side", [0, 1])
def test_graded_spectrum_ket_is_orthonormal(ctx, side):
    """Sector matrices with singular values spread from 1 down to 1e-13 (the
    kept ones reach the canpre cut): the Jacobi convergence test leaves the
    working matrix's columns of such tiny values non-orthogonal by up to
    eps ||A|| / s, so the new ket is orthonormalised and the canonical block is
    the projection of A on it.  Checked against numpy's SVD: the ket
    orthonormal within 1e-12, the kept singular values (canonical row / column
    norms) and the truncated product (ket x canonical) within 1e-12 of
    ||A||, the truncation dimensions equal."""
    rng = np.random.default_rng(11)
    shapes = [(300, 120), (250, 64), (90, 40)] if side == 0 else [(120, 300), (64, 250), (40, 90)]
    A = []
    for m, n in shapes:
        k = min(m, n)
        U, _ = np.linalg.qr(rng.standard_normal((m, k)))
        V, _ = np.linalg.qr(rng.standard_normal((n, k)))
        s = np.logspace(0, -13, k) * rng.uniform(0.5, 1.0)
        A.append((U * s) @ V.T)
    ns = len(A)
    m = np.array([a.shape[0] for a in A])
    n = np.array([a.shape[1] for a in A])
    ket = capi.BlockSpec(np.arange(ns), np.arange(ns), m, n)
    c = capi.Canonical(ctx, side, m, n, ket)
    kdev = capi.DeviceArray.from_host(ctx, np.concatenate([a.ravel() for a in A]))
    canpre = 1e-12
    res = c.run(kdev, 10000, canpre)
    newk = capi.DeviceArray(ctx, res["ket_size"])
    can = capi.DeviceArray(ctx, res["canonical_size"])
    c.write(kdev, newk, can)
    ctx.sync()
    K, Cn = newk.download(), can.download()
    kp = cp = 0
    for i, a in enumerate(A):
        Ur, sr, Vtr = np.linalg.svd(a, full_matrices=False)
        t = int((sr > canpre).sum())
        assert res["tdim"][i] == t
        kr, kc = res["ket_rows"][i], res["ket_cols"][i]
        Kb = K[kp:kp + kr * kc].reshape(kr, kc)
        kp += kr * kc
        cr, cc = res["canon_rows"][i], res["canon_cols"][i]
        Cb = Cn[cp:cp + cr * cc].reshape(cr, cc)
        cp += cr * cc
        gram = Kb.T @ Kb if side == 0 else Kb @ Kb.T
        assert np.abs(gram - np.eye(t)).max() < 1e-12
        norms = np.linalg.norm(Cb, axis=1 if side == 0 else 0)
        assert np.abs(norms - sr[:t]).max() < 1e-12
        prod = Kb @ Cb if side == 0 else Cb @ Kb
        ref = (Ur[:, :t] * sr[:t]) @ Vtr[:t]
        assert np.abs(prod - ref).max() < 1e-12
