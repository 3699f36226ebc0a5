"""Config-scale parity: environment updates, canonicalisations and a Lanczos
solve at bond dimension 1024 on the 8x4 cylinder (d=5, N=16, U=8),
against the reference's own outputs (tests/golden/make_golden.py --d1024).

* Environment updates (left at site 4, right at site 27) and canonicalisations
  (left at site 6, right at site 25, both on the subspace-expanded tensor with
  ragged blocks) use the reference's block structures at that point of its run
  and seeded synthetic values (the reference ran on the same values,
  PROBE_SYNTH): output block maps bit-exact; sampled output entries within
  1e-12 of the largest (environments) and 1e-11 (the gauge-invariant products
  U S V^T of the canonicalisation); singular values within 1e-12 of the
  largest; truncation dimensions bit-exact.
* The Lanczos solve (site 4, psi_dim ~67k, its environments as the reference
  had them, rounded to float32 before the reference solved): energy within
  1e-12 per site, overlap with the reference's ground vector 1 - 1e-7 (the
  numpy oracle itself sits at 1 - 1.8e-8 from it: at this site the Lanczos
  vector is converged only to a residual of 2e-6, so rounding-level
  differences move it further than the chain16 fixtures' 1e-9 bar)."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from dmrgcc_b200.problem import read_nac

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _spec(d, p):
    return capi.BlockSpec(d[p + ".left"], d[p + ".right"], d[p + ".rows"], d[p + ".cols"])


def _site(d, p="lattice"):
    nl, nr = len(d[p + ".left_dim"]), len(d[p + ".right_dim"])
    dd, lb, rb = (int(x) for x in d["op.dims"])
    W = np.asarray(d["op.W"], dtype=np.float64).reshape(lb, rb, dd, dd)
    return capi.SiteProblem(nl, nr, d[p + ".physics_index"], _spec(d, p + ".ket"), W)


@pytest.mark.parametrize("call", [283, 314])
def test_env_update_D1024_matches_reference(ctx, call):
    d = read_nac(os.path.join(GOLD, f"env_cyl8x4_D1024_c{call}.nac"))
    side = 0 if d["left"][0] else 1
    seed = int(d["synth_seed"][0])
    site = _site(d)
    nin, nout = int(d["env_in.bond"][0]), int(d["env_out.bond"][0])
    e = capi.Env(ctx, side, site, [_spec(d, f"env_in.{o}") for o in range(nin)])
    assert e.out_bond == nout
    for o, blk in enumerate(e.out_blocks()):
        for f in ("left", "right", "rows", "cols"):
            assert np.array_equal(getattr(blk, f), d[f"env_out.{o}.{f}"]), (o, f)
    psi_dim = site.ket.size
    n_in = sum(_spec(d, f"env_in.{o}").size for o in range(nin))
    ket = capi.DeviceArray(ctx, psi_dim)
    ket.fill_uniform(seed, 0)
    ein = capi.DeviceArray(ctx, n_in)
    ein.fill_uniform(seed, psi_dim)
    eout = capi.DeviceArray(ctx, e.out_size)
    e.apply(ket, ein, eout)
    ctx.sync()
    got = eout.download()
    idx, ref = d["digest.index"], np.asarray(d["digest.value"])
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(got[idx] - ref)) <= 1e-12 * scale
    sizes = [_spec(d, f"env_out.{o}").size for o in range(nout)]
    parts = np.split(got, np.cumsum(sizes)[:-1])
    sumsq = np.array([float(np.sum(x * x)) for x in parts])
    assert np.allclose(sumsq, d["digest.sumsq"], rtol=1e-12, atol=1e-12 * float(np.max(d["digest.sumsq"])))


@pytest.mark.parametrize("call", [318, 349])
def test_canonicalisation_D1024_matches_reference(ctx, call):
    d = read_nac(os.path.join(GOLD, f"canon_cyl8x4_D1024_c{call}.nac"))
    left = bool(d["left"][0])
    side = 0 if left else 1
    seed = int(d["synth_seed"][0])
    ket = _spec(d, "before.ket")
    c = capi.Canonical(ctx, side, d["before.left_dim"], d["before.right_dim"], ket)
    kdev = capi.DeviceArray(ctx, ket.size)
    kdev.fill_uniform(seed, 0)
    res = c.run(kdev, int(d["max_dim"][0]), float(d["canpre"][0]))
    ref_dims = d["after.right_dim"] if left else d["after.left_dim"]
    assert np.array_equal(res["tdim"], ref_dims)
    assert np.array_equal(res["ket_rows"], d["after.ket.rows"])
    assert np.array_equal(res["ket_cols"], d["after.ket.cols"])
    assert np.array_equal(res["canon_rows"], d["after.canonical.rows"])
    assert np.array_equal(res["canon_cols"], d["after.canonical.cols"])
    assert np.array_equal(res["match_dim"], d["after.match_dim"])
    # singular values of every sector (the kept ones are in the reference's S).
    # A sector whose kept block the truncation forces to zero (one row of zeros in
    # the reference's S V^T) reports its raw values here; its zero output is
    # checked by the gauge-invariant products below.
    counts, sig = d["digest.sigma_count"], np.asarray(d["digest.sigma"])
    smax = float(np.max(sig))
    off = 0
    forced = 0
    for s, n in enumerate(counts):
        ref = np.sort(sig[off:off + n])[::-1]
        off += n
        if n and not np.any(ref):
            forced += 1
            continue
        got = c.singular_values(s)[:n]
        assert np.max(np.abs(np.sort(got)[::-1] - ref), initial=0.0) <= 1e-12 * smax
    assert forced < len(counts)
    # gauge-invariant products: new ket block x canonical block of its sector
    newk = capi.DeviceArray(ctx, res["ket_size"])
    can = capi.DeviceArray(ctx, res["canonical_size"])
    c.write(kdev, newk, can)
    ctx.sync()
    kd, cd = newk.download(), can.download()
    kr, kc = res["ket_rows"], res["ket_cols"]
    cr, cc = res["canon_rows"], res["canon_cols"]
    koff = np.concatenate([[0], np.cumsum(kr.astype(np.int64) * kc)])
    coff = np.concatenate([[0], np.cumsum(cr.astype(np.int64) * cc)])
    prods = []
    for k in range(len(kr)):
        b = kd[koff[k]:koff[k + 1]].reshape(kr[k], kc[k])
        s = d["after.ket.right"][k] if left else d["after.ket.left"][k]
        m = cd[coff[s]:coff[s + 1]].reshape(cr[s], cc[s])
        prods.append((b @ m if left else m @ b).ravel())
    flat = np.concatenate(prods)
    idx, ref = d["digest.index"], np.asarray(d["digest.value"])
    assert np.max(np.abs(flat[idx] - ref)) <= 1e-11 * np.max(np.abs(ref))
    assert abs(float(np.sum(flat * flat)) - float(d["digest.prod_sumsq"][0])) <= 1e-11 * float(d["digest.prod_sumsq"][0])


def test_lanczos_D1024_matches_reference(ctx):
    z = np.load(os.path.join(GOLD, "lanczos_cyl8x4_D1024_c252.npz"))
    d = {k: z[k] for k in z.files}
    site = _site(d)
    dd, lb, rb = (int(x) for x in d["op.dims"])
    L = [_spec(d, f"L.{o}") for o in range(lb)]
    R = [_spec(d, f"R.{o}") for o in range(rb)]
    cat = lambda p, n: np.concatenate([np.asarray(d[f"{p}.{o}.data"], np.float64) for o in range(n)])
    h = capi.Heff(ctx, site, L, R)
    Ld = capi.DeviceArray.from_host(ctx, cat("L", lb))
    Rd = capi.DeviceArray.from_host(ctx, cat("R", rb))
    h.set_env(Ld, Rd)
    psi = capi.DeviceArray.from_host(ctx, np.asarray(d["lattice.ket.data"], np.float64))
    e, dim = h.lanczos(psi, int(d["niter"][0]))
    assert abs(e - float(d["energy"][0])) / 32 <= 1e-12
    v = psi.download()
    g = np.asarray(d["ground"], np.float64)
    g /= np.linalg.norm(g)
    assert 1.0 - abs(float(v @ g)) <= 1e-7
    assert 1 <= dim <= int(d["niter"][0])


@pytest.mark.parametrize("call", [283, 314])
@pytest.mark.parametrize("prec,tol", [(capi.DMRG_PREC_TF32X3, 2e-5), (capi.DMRG_PREC_BF16X3, 2e-4)])
def test_env_update_D1024_split_precision(ctx, call, prec, tol):
    """The same D=1024 environment updates with split-precision products on the
    tensor cores (tcgen05; hi/lo parts, FP32 accumulation per product, FP64
    sums): same block maps, values within `tol` of the largest FP64 entry."""
    d = read_nac(os.path.join(GOLD, f"env_cyl8x4_D1024_c{call}.nac"))
    side = 0 if d["left"][0] else 1
    seed = int(d["synth_seed"][0])
    site = _site(d)
    nin = int(d["env_in.bond"][0])
    specs = [_spec(d, f"env_in.{o}") for o in range(nin)]
    ket = capi.DeviceArray(ctx, site.ket.size)
    ket.fill_uniform(seed, 0)
    ein = capi.DeviceArray(ctx, sum(s.size for s in specs))
    ein.fill_uniform(seed, site.ket.size)
    outs = []
    for p in (capi.DMRG_PREC_FP64, prec):
        e = capi.Env(ctx, side, site, specs, precision=p)
        eout = capi.DeviceArray(ctx, e.out_size)
        for _ in range(2):  # repeated applications overwrite
            e.apply(ket, ein, eout)
        ctx.sync()
        outs.append(eout.download())
    ref, got = outs
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) <= tol * np.max(np.abs(ref))
    assert np.max(np.abs(got - ref)) > 0.0  # the split path did run
