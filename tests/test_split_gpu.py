"""Split-precision H_eff*psi (DMRG_PREC_TF32X3, tcgen05 tensor cores with TF32
hi/lo splits and FP32 accumulation) against the FP64 path on the same operator
and vectors.  The products drop the lo*lo term (~2^-22 relative) and round each
operand to FP32 first, and the block sums accumulate in FP32, so the bound is
relative to the largest output: max |TF32X3 - FP64| <= 2e-5 * max |FP64|."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from dmrgcc_b200.problem import SiteStep

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 2e-5


def _pair(ctx, step, L, R):
    hs = []
    for prec in (capi.DMRG_PREC_FP64, capi.DMRG_PREC_TF32X3):
        h = capi.Heff(ctx, step.site, step.L, step.R, precision=prec)
        h.set_env(L, R)
        hs.append(h)
    return hs


def _compare(ctx, h64, h3, psi, n):
    outs = []
    for h in (h64, h3):
        out = capi.DeviceArray(ctx, n)
        out.upload(np.full(n, 3.0))  # overwritten (accumulate=False)
        h.apply(psi, out, accumulate=False)
        ctx.sync()  # also reports a tensor-core wait that gave up
        outs.append(out.download())
    ref, got = outs
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    return ref, got, err


def test_tf32x3_heff_matches_fp64_on_reference_operator(ctx):
    step = SiteStep.from_nac(os.path.join(GOLD, "heff_c158.nac"))
    L = capi.DeviceArray.from_host(ctx, step.L_data)
    R = capi.DeviceArray.from_host(ctx, step.R_data)
    h64, h3 = _pair(ctx, step, L, R)
    psi = capi.DeviceArray.from_host(ctx, step.ket_data)
    ref, got, err = _compare(ctx, h64, h3, psi, step.psi_dim)
    assert err <= TOL, err
    assert err > 0.0  # it really ran in reduced precision
    # accumulate adds into the output like the FP64 path
    out = capi.DeviceArray.from_host(ctx, ref)
    h3.apply(psi, out, accumulate=True)
    ctx.sync()
    assert np.max(np.abs(out.download() - 2 * ref)) <= 2 * TOL * np.max(np.abs(ref))


def test_tf32x3_heff_matches_fp64_at_d1024(ctx):
    step = SiteStep.from_nac(os.path.join(GOLD, "heff_struct_cyl8x4_D1024.nac"))
    psi, L, R = step.synthetic_device(ctx, seed=11)
    h64, h3 = _pair(ctx, step, L, R)
    ref, got, err = _compare(ctx, h64, h3, psi, step.psi_dim)
    assert err <= TOL, err
    # the same rounding every call (fixed summation order)
    _, got2, _ = _compare(ctx, h64, h3, psi, step.psi_dim)
    assert np.array_equal(got, got2)


@pytest.mark.parametrize("call", [20, 158])
def test_mixed_precision_lanczos_matches_reference(ctx, call):
    """A DMRG_PREC_TF32X3 operator runs the Lanczos first on split-precision
    matvecs, then the FP64 Lanczos from that vector: the energy and the state
    meet the FP64 parity bar (|dE|/site <= 1e-12, overlap 1 - 1e-9)."""
    from dmrgcc_b200.problem import read_nac
    step = SiteStep.from_nac(os.path.join(GOLD, f"heff_c{call}.nac"))
    ref = read_nac(os.path.join(GOLD, f"lanczos_c{call}.nac"))
    niter = int(read_nac(os.path.join(GOLD, f"heff_c{call}.nac"))["niter"][0])
    L = capi.DeviceArray.from_host(ctx, step.L_data)
    R = capi.DeviceArray.from_host(ctx, step.R_data)
    h = capi.Heff(ctx, step.site, step.L, step.R, precision=capi.DMRG_PREC_TF32X3)
    h.set_env(L, R)
    psi = capi.DeviceArray.from_host(ctx, step.ket_data)
    e, dim = h.lanczos(psi, niter)
    assert abs(e - float(ref["energy"][0])) / 16 <= 1e-12
    v = psi.download()
    assert 1.0 - abs(float(v @ np.asarray(ref["lattice.ket.data"]))) <= 1e-9
