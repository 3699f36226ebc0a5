"""Split-precision H_eff*psi on the tcgen05 tensor cores against the FP64 path
on the same operator and vectors.  DMRG_PREC_TF32X3 (TF32 hi/lo parts of each
operand rounded to FP32, FP32 accumulation per term): max |split - FP64| <=
2e-5 * max |FP64|.  DMRG_PREC_BF16X3 (bf16 hi/lo parts, ~16 bits per operand):
<= 2e-4 * max |FP64|.  Both drop the lo*lo product and add the terms of a block
sum in FP64."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from dmrgcc_b200.problem import SiteStep

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOLS = {capi.DMRG_PREC_TF32X3: 2e-5, capi.DMRG_PREC_BF16X3: 2e-4}
SPLITS = [capi.DMRG_PREC_TF32X3, capi.DMRG_PREC_BF16X3]


def _pair(ctx, step, L, R, split):
    hs = []
    for prec in (capi.DMRG_PREC_FP64, split):
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


@pytest.mark.parametrize("split", SPLITS)
def test_split_heff_matches_fp64_on_reference_operator(ctx, split):
    TOL = TOLS[split]
    step = SiteStep.from_nac(os.path.join(GOLD, "heff_c158.nac"))
    L = capi.DeviceArray.from_host(ctx, step.L_data)
    R = capi.DeviceArray.from_host(ctx, step.R_data)
    h64, h3 = _pair(ctx, step, L, R, split)
    psi = capi.DeviceArray.from_host(ctx, step.ket_data)
    ref, got, err = _compare(ctx, h64, h3, psi, step.psi_dim)
    assert err <= TOL, err
    assert err > 0.0  # it really ran in reduced precision
    # accumulate adds into the output like the FP64 path
    out = capi.DeviceArray.from_host(ctx, ref)
    h3.apply(psi, out, accumulate=True)
    ctx.sync()
    assert np.max(np.abs(out.download() - 2 * ref)) <= 2 * TOL * np.max(np.abs(ref))


@pytest.mark.parametrize("split", SPLITS)
def test_split_heff_matches_fp64_at_d1024(ctx, split):
    TOL = TOLS[split]
    step = SiteStep.from_nac(os.path.join(GOLD, "heff_struct_cyl8x4_D1024.nac"))
    psi, L, R = step.synthetic_device(ctx, seed=11)
    h64, h3 = _pair(ctx, step, L, R, split)
    ref, got, err = _compare(ctx, h64, h3, psi, step.psi_dim)
    assert err <= TOL, err
    # the same rounding every call (fixed summation order)
    _, got2, _ = _compare(ctx, h64, h3, psi, step.psi_dim)
    assert np.array_equal(got, got2)


@pytest.mark.parametrize("split", SPLITS)
@pytest.mark.parametrize("call", [20, 158])
@pytest.mark.parametrize("polish,de_tol,ov_tol", [(0, 1e-12, 1e-9), (4, 1e-10, 1e-7)])
def test_mixed_precision_lanczos_matches_reference(ctx, call, split, polish, de_tol, ov_tol):
    """A split-precision operator runs the Lanczos first on split-precision
    matvecs, then an FP64 Krylov run from that vector.  The full FP64 Lanczos
    (polish 0) meets the FP64 parity bar (|dE|/site <= 1e-12, overlap 1 - 1e-9);
    the default short run of 4 FP64 matvecs meets |dE|/site <= 1e-10 (the
    split mode's target) and overlap 1 - 1e-7."""
    from dmrgcc_b200.problem import read_nac
    step = SiteStep.from_nac(os.path.join(GOLD, f"heff_c{call}.nac"))
    ref = read_nac(os.path.join(GOLD, f"lanczos_c{call}.nac"))
    niter = int(read_nac(os.path.join(GOLD, f"heff_c{call}.nac"))["niter"][0])
    L = capi.DeviceArray.from_host(ctx, step.L_data)
    R = capi.DeviceArray.from_host(ctx, step.R_data)
    h = capi.Heff(ctx, step.site, step.L, step.R, precision=split)
    h.set_env(L, R)
    h.set_split_threshold(0)  # the mixed path at any size (the default keeps it for large psi_dim)
    psi = capi.DeviceArray.from_host(ctx, step.ket_data)
    lib = capi.lib()
    try:
        assert lib.dmrg_lanczos_set_polish(polish) == 0
        e, dim = h.lanczos(psi, niter)
    finally:
        lib.dmrg_lanczos_set_polish(4)
    assert h.split_iters() > 0
    assert abs(e - float(ref["energy"][0])) / 16 <= de_tol
    v = psi.download()
    assert 1.0 - abs(float(v @ np.asarray(ref["lattice.ket.data"]))) <= ov_tol


@pytest.mark.parametrize("split", SPLITS)
def test_split_operator_small_problem_runs_fp64_lanczos(ctx, split):
    """Below the split threshold (default psi_dim 200000) a split-precision
    operator's Lanczos is the FP64 one: same dimension, energy and vector."""
    from dmrgcc_b200.problem import read_nac
    step = SiteStep.from_nac(os.path.join(GOLD, "heff_c158.nac"))
    niter = int(read_nac(os.path.join(GOLD, "heff_c158.nac"))["niter"][0])
    L = capi.DeviceArray.from_host(ctx, step.L_data)
    R = capi.DeviceArray.from_host(ctx, step.R_data)
    res = []
    for prec in (capi.DMRG_PREC_FP64, split):
        h = capi.Heff(ctx, step.site, step.L, step.R, precision=prec)
        h.set_env(L, R)
        psi = capi.DeviceArray.from_host(ctx, step.ket_data)
        res.append(h.lanczos(psi, niter) + (psi.download(),))
        assert h.split_iters() == 0
    (e0, d0, v0), (e1, d1, v1) = res
    assert d0 == d1 and e0 == e1 and np.array_equal(v0, v1)
