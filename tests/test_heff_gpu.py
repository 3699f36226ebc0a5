"""a1 parity: the sm_100a H_eff*psi against the reference's own outputs and the
oracle.  FP64 tolerance: max |GPU - ref| <= 1e-12 * max |ref| (different, but
fixed, summation order)."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from dmrgcc_b200.problem import SiteStep
from oracle import dmrg_oracle as O
from oracle.nac import read_nac

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-12


def _heff_from_fixture(ctx, name):
    step = SiteStep.from_nac(os.path.join(GOLD, name))
    h = capi.Heff(ctx, step.site, step.L, step.R)
    L = capi.DeviceArray.from_host(ctx, step.L_data)
    R = capi.DeviceArray.from_host(ctx, step.R_data)
    h.set_env(L, R)
    return step, h, (L, R)


@pytest.mark.parametrize("name", ["heff_c20.nac", "heff_c158.nac"])
def test_heff_matches_reference_output(ctx, name):
    step, h, keep = _heff_from_fixture(ctx, name)
    ref = read_nac(os.path.join(GOLD, name))["heff_out"]
    psi = capi.DeviceArray.from_host(ctx, step.ket_data)
    out = capi.DeviceArray(ctx, step.psi_dim)
    h.apply(psi, out, accumulate=False)
    ctx.sync()
    got = out.download()
    assert np.max(np.abs(got - ref)) <= TOL * np.max(np.abs(ref))
    alg, exe = h.flops()
    assert alg > 0 and exe <= alg * 1.0000001


def test_heff_accumulates_like_reference(ctx):
    # The reference adds into `state` (state[part_dim + a] +=); accumulate=True too.
    step, h, keep = _heff_from_fixture(ctx, "heff_c158.nac")
    ref = read_nac(os.path.join(GOLD, "heff_c158.nac"))["heff_out"]
    base = np.linspace(-1, 1, step.psi_dim)
    psi = capi.DeviceArray.from_host(ctx, step.ket_data)
    out = capi.DeviceArray.from_host(ctx, base)
    h.apply(psi, out, accumulate=True)
    ctx.sync()
    assert np.max(np.abs(out.download() - (base + ref))) <= TOL * np.max(np.abs(ref))
    # host-buffer entry point, twice in a row
    host_out = base.copy()
    h.apply_host(np.ascontiguousarray(step.ket_data), host_out, accumulate=True)
    h.apply_host(np.ascontiguousarray(step.ket_data), host_out, accumulate=True)
    assert np.max(np.abs(host_out - (base + 2 * ref))) <= TOL * np.max(np.abs(ref))


def test_fill_uniform_matches_oracle_stream(ctx):
    a = capi.DeviceArray(ctx, 1000)
    a.fill_uniform(99, 12345)
    ctx.sync()
    assert np.array_equal(a.download(), O.splitmix_uniform(99, 12345, 1000))


def test_heff_cylinder_D1024_synthetic(ctx):
    """Full-size structure (8x4 cylinder, D=1024, site 16, dumped from the reference)
    with seeded values: GPU vs the oracle on the same values."""
    path = os.path.join(GOLD, "heff_struct_cyl8x4_D1024.nac")
    step = SiteStep.from_nac(path)
    h = capi.Heff(ctx, step.site, step.L, step.R)
    psi, L, R = step.synthetic_device(ctx, seed=2024)
    h.set_env(L, R)
    out = capi.DeviceArray(ctx, step.psi_dim)
    h.apply(psi, out)
    ctx.sync()
    got = out.download()

    d = read_nac(path)
    lat = O.lattice_from_nac(d, "lattice")
    W = O.operator_from_nac(d, "op")
    Lo, Ro = O.env_from_nac(d, "L"), O.env_from_nac(d, "R")
    vals = O.splitmix_uniform(2024, 0, step.psi_dim + step.l_size + step.r_size)
    lat.ket.unvectorize(vals[:step.psi_dim])
    pos = step.psi_dim
    for env in (Lo, Ro):
        for blk in env:
            for i, m in enumerate(blk.mats):
                blk.mats[i] = vals[pos:pos + m.size].reshape(m.shape).copy()
                pos += m.size
    ref = np.zeros(step.psi_dim)
    O.multiply_effect_hamilton(lat, W, Lo, Ro, ref)
    assert np.max(np.abs(got - ref)) <= TOL * np.max(np.abs(ref))
    fa, fb = O.heff_flops(lat, W, Lo, Ro)
    alg, _ = h.flops()
    assert abs(alg - (fa + fb)) <= 1e-9 * alg
