"""Batched one-sided Jacobi SVD (a6) on synthetic sectors of edge shapes, in one
canonicalisation call: 1x1, tall and wide blocks, sizes around the 32-column
block and 64-column pair boundaries and the Gram items' 64-row ranges, with
graded singular values 1 ... 1e-13 (each sector has one block, so its singular
values are those of the block).  Checked against numpy's SVD of the same
matrices: singular values to 1e-13 of the largest; U * canonical (S V^T) equal
to the input to 1e-12; the columns of U of unit norm, and mutually orthogonal
to the one-sided Jacobi's stopping rule, which is backward stable (absolute):
|(u_i s_i) . (u_j s_j)| <= 1e-13 s_max^2, so that a column of tiny s_i is
orthogonal only to ~eps s_max / s_i (dgesvd's U would be orthonormal to eps)."""
import numpy as np
import pytest

from dmrgcc_b200 import capi

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1), (5, 3), (3, 5), (31, 17), (63, 40), (64, 64), (65, 33), (97, 96), (130, 129), (200, 65),
          (40, 300), (300, 200)]


def _graded(rng, m, n):
    k = min(m, n)
    u, _ = np.linalg.qr(rng.standard_normal((m, k)))
    v, _ = np.linalg.qr(rng.standard_normal((n, k)))
    sigma = np.logspace(0, -13, k) if k > 1 else np.ones(1)
    return (u * sigma) @ v.T


def test_batched_svd_on_edge_shapes(ctx):
    rng = np.random.default_rng(7)
    mats = [_graded(rng, m, n) for m, n in SHAPES]
    ns = len(SHAPES)
    idx = np.arange(ns, dtype=np.int32)
    rows = np.array([m for m, _ in SHAPES], dtype=np.int32)
    cols = np.array([n for _, n in SHAPES], dtype=np.int32)
    ket = capi.BlockSpec(idx, idx, rows, cols)
    c = capi.Canonical(ctx, 0, rows, cols, ket)
    kdev = capi.DeviceArray.from_host(ctx, np.concatenate([a.ravel() for a in mats]))
    res = c.run(kdev, 10**6, 1e-300)
    for s, a in enumerate(mats):
        ref = np.linalg.svd(a, compute_uv=False)
        got = np.sort(c.singular_values(s))[::-1]
        assert got.shape == ref.shape, f"sector {s} {SHAPES[s]}"
        assert np.max(np.abs(got - ref)) <= 1e-13 * ref[0], f"sector {s} {SHAPES[s]}"
    newk = capi.DeviceArray(ctx, res["ket_size"])
    can = capi.DeviceArray(ctx, res["canonical_size"])
    c.write(kdev, newk, can)
    ctx.sync()
    K, Cn = newk.download(), can.download()
    kp = cp = 0
    for s, a in enumerate(mats):
        kr, kc = int(res["ket_rows"][s]), int(res["ket_cols"][s])
        cr, cc = int(res["canon_rows"][s]), int(res["canon_cols"][s])
        u = K[kp:kp + kr * kc].reshape(kr, kc)
        sv = Cn[cp:cp + cr * cc].reshape(cr, cc)
        kp += kr * kc
        cp += cr * cc
        assert kr == a.shape[0] and kc == min(a.shape), f"sector {s} {SHAPES[s]}"
        sig = np.linalg.norm(sv, axis=1)  # the canonical block is S V^T: its row norms are the s_i
        assert np.allclose(np.linalg.norm(u, axis=0), 1.0, rtol=0, atol=1e-12), f"sector {s} {SHAPES[s]}"
        w = u * sig
        off = w.T @ w - np.diag(sig * sig)
        assert np.max(np.abs(off)) <= 1e-13 * sig.max() ** 2, f"sector {s} {SHAPES[s]}"
        assert np.allclose(u @ sv, a, rtol=0, atol=1e-12), f"sector {s} {SHAPES[s]}"


def test_batched_svd_on_tiny_sectors(ctx):
    """Sectors whose entries lie near 1e-80 .. 1e-117 (a state's negligible
    sectors; tests/golden/svd_tiny_sectors.npz holds two from the U/t scan's
    32-site chain, on which an unscaled Jacobi never converged because the
    squared thresholds underflowed) and graded matrices scaled by 1e-95: the
    sweeps converge, singular values match numpy's to 1e-13 of the largest and
    U * (S V^T) reproduces the input to 1e-12 of its norm."""
    import os

    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "svd_tiny_sectors.npz"))
    rng = np.random.default_rng(11)
    mats = [z[k] for k in sorted(z.files)] + [0.7e-95 * _graded(rng, m, n) for m, n in ((40, 30), (20, 70))]
    ns = len(mats)
    idx = np.arange(ns, dtype=np.int32)
    rows = np.array([a.shape[0] for a in mats], dtype=np.int32)
    cols = np.array([a.shape[1] for a in mats], dtype=np.int32)
    ket = capi.BlockSpec(idx, idx, rows, cols)
    c = capi.Canonical(ctx, 0, rows, cols, ket)
    kdev = capi.DeviceArray.from_host(ctx, np.concatenate([a.ravel() for a in mats]))
    res = c.run(kdev, 10**6, 1e-300)
    for s, a in enumerate(mats):
        ref = np.linalg.svd(a, compute_uv=False)
        got = np.sort(c.singular_values(s))[::-1]
        assert np.max(np.abs(got - ref)) <= 1e-13 * ref[0], f"sector {s}"
    newk = capi.DeviceArray(ctx, res["ket_size"])
    can = capi.DeviceArray(ctx, res["canonical_size"])
    c.write(kdev, newk, can)
    ctx.sync()
    K, Cn = newk.download(), can.download()
    kp = cp = 0
    for s, a in enumerate(mats):
        kr, kc = int(res["ket_rows"][s]), int(res["ket_cols"][s])
        cr, cc = int(res["canon_rows"][s]), int(res["canon_cols"][s])
        u = K[kp:kp + kr * kc].reshape(kr, kc)
        sv = Cn[cp:cp + cr * cc].reshape(cr, cc)
        kp += kr * kc
        cp += cr * cc
        assert np.linalg.norm(u @ sv - a) <= 1e-12 * np.linalg.norm(a), f"sector {s}"
