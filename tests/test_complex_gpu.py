"""The complex path on the device against the reference's complex DMRG
(Bose-Hubbard-Hofstadter on a 4x3 cylinder, flux 1/6: the reference's spinful
executable with Ndown = 0, tests/golden/make_golden.py --complex):

* complex H_eff*psi (dmrg_zheff_apply: four real DMMA products per complex
  product) against ComplexTensorContraction::MultiplyEffectHamilton's output:
  1e-12 of the largest entry;
* the complex Lanczos (dmrg_zlanczos, conjugated inner products) against
  ComplexTensorLanczos::LanczosMethod: energy within 1e-12 per MPS site, the
  ground vector equal up to a global phase (|<psi|psi_ref>| = 1 - 1e-9), for a
  Krylov case (psi_dim 313) and the dense branch (psi_dim 54)."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from dmrgcc_b200.problem import read_nac

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
N_SITES = 24


def _spec(d, p):
    return capi.BlockSpec(d[p + ".left"], d[p + ".right"], d[p + ".rows"], d[p + ".cols"])


def _problem(ctx, call):
    d = read_nac(os.path.join(GOLD, f"zheff_hof_c{call}.nac"))
    nl, nr = len(d["lattice.left_dim"]), len(d["lattice.right_dim"])
    dd, lb, rb = (int(x) for x in d["op.dims"])
    Wc = np.asarray(d["op.W"]).view(np.complex128).reshape(lb, rb, dd, dd)
    site = capi.SiteProblem(nl, nr, d["lattice.physics_index"], _spec(d, "lattice.ket"), Wc.real)
    L = [_spec(d, f"L.{o}") for o in range(lb)]
    R = [_spec(d, f"R.{o}") for o in range(rb)]
    h = capi.ZHeff(ctx, site, L, R, Wc)
    cat = lambda p, n: np.concatenate([np.asarray(d[f"{p}.{o}.data"]) for o in range(n)])
    Ld = capi.DeviceArray.from_host(ctx, cat("L", lb))
    Rd = capi.DeviceArray.from_host(ctx, cat("R", rb))
    h.set_env(Ld, Rd)
    return d, h, (Ld, Rd)


@pytest.mark.parametrize("call", [182, 196])
def test_complex_heff_matches_reference(ctx, call):
    d, h, keep = _problem(ctx, call)
    psi = capi.DeviceArray.from_host(ctx, np.asarray(d["lattice.ket.data"]))
    out = capi.DeviceArray(ctx, 2 * h.psi_dim)
    out.upload(np.full(2 * h.psi_dim, 3.0))  # overwritten (accumulate = 0)
    h.apply(psi, out)
    ctx.sync()
    got = out.download().view(np.complex128)
    ref = np.asarray(d["heff_out"]).view(np.complex128)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    h.apply(psi, out, accumulate=True)  # adds like the reference's state +=
    ctx.sync()
    assert np.max(np.abs(out.download().view(np.complex128) - 2 * ref)) <= 2e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("call", [182, 196])
def test_complex_lanczos_matches_reference(ctx, call):
    d, h, keep = _problem(ctx, call)
    ref = read_nac(os.path.join(GOLD, f"zlanczos_hof_c{call}.nac"))
    psi = capi.DeviceArray.from_host(ctx, np.asarray(d["lattice.ket.data"]))
    e, dim = h.lanczos(psi, int(d["niter"][0]))
    assert abs(e - float(ref["energy"][0])) / N_SITES <= 1e-12
    v = psi.download().view(np.complex128)
    v_ref = np.asarray(ref["lattice.ket.data"]).view(np.complex128)
    assert abs(np.linalg.norm(v) - 1.0) <= 1e-10
    assert 1.0 - abs(np.vdot(v_ref, v)) / np.linalg.norm(v_ref) <= 1e-9
    if h.psi_dim < 100:
        assert dim == 0
    else:
        assert 1 <= dim <= int(d["niter"][0])
    # an eigenvector of the complex operator
    out = capi.DeviceArray(ctx, 2 * h.psi_dim)
    h.apply(psi, out)
    ctx.sync()
    r = out.download().view(np.complex128) - e * v
    assert np.linalg.norm(r) <= 1e-6 * max(1.0, abs(e))
