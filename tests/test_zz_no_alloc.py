"""dmrg_heff_apply_noalloc: H_eff * psi for callers that cannot allocate device
memory (for example a host framework that owns every device allocation under a
fixed budget).  It must agree with the allocating entry point dmrg_heff_apply,
within the H_eff tolerance used elsewhere (1e-12 relative), on two calls in a row
(the static scratch keeps the previous call's contents), and reject a problem
whose schedule does not fit its 16 MiB static scratch with a clear error.

Collected last on purpose (file name): if it fails, every other test has run."""
import ctypes as C
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from dmrgcc_b200.problem import SiteStep, read_nac

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-12


def _noalloc(step, Lb, Rb, L, R, psi, out, accumulate, stream):
    site = step.site
    kb = site.ket.c()
    return capi.lib().dmrg_heff_apply_noalloc(
        site.nl, site.nr, site.phys.ctypes.data_as(C.POINTER(C.c_int)), C.byref(kb), site.d, site.lb, site.rb,
        site.W.ctypes.data_as(C.POINTER(C.c_double)), Lb, Rb, L.ptr, R.ptr, psi.ptr, out.ptr, int(accumulate), stream)


def _blocks(specs):
    arr = (capi.Blocks * len(specs))()
    for i, s in enumerate(specs):
        arr[i] = s.c()
    return arr


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point():
    ctx = capi.Context(0)
    step = SiteStep.from_nac(os.path.join(GOLD, "heff_c158.nac"))
    L = capi.DeviceArray.from_host(ctx, step.L_data)
    R = capi.DeviceArray.from_host(ctx, step.R_data)
    psi = capi.DeviceArray.from_host(ctx, step.ket_data)
    # the existing entry point
    h = capi.Heff(ctx, step.site, step.L, step.R)
    h.set_env(L, R)
    ref = capi.DeviceArray(ctx, step.psi_dim)
    h.apply(psi, ref)
    ctx.sync()
    want = ref.download()
    scale = np.max(np.abs(want))
    Lb, Rb = _blocks(step.L), _blocks(step.R)
    out = capi.DeviceArray(ctx, step.psi_dim)
    for call in range(2):  # two calls in a row share the static scratch
        out.upload(np.full(step.psi_dim, 7.0))  # overwritten (accumulate = 0)
        rc = _noalloc(step, Lb, Rb, L, R, psi, out, False, ctx.stream)
        assert rc == 0, capi.lib().dmrg_last_error()
        ctx.sync()
        assert np.max(np.abs(out.download() - want)) <= TOL * scale, f"call {call}"
    # accumulate = 1 adds into out, like the reference's state +=
    rc = _noalloc(step, Lb, Rb, L, R, psi, out, True, ctx.stream)
    assert rc == 0
    ctx.sync()
    assert np.max(np.abs(out.download() - 2 * want)) <= 2 * TOL * scale
    # the allocating entry point's own output: the reference's heff_out (1e-12)
    ref_out = np.asarray(read_nac(os.path.join(GOLD, "heff_c158.nac"))["heff_out"])
    out.upload(np.zeros(step.psi_dim))
    assert _noalloc(step, Lb, Rb, L, R, psi, out, False, ctx.stream) == 0
    ctx.sync()
    assert np.max(np.abs(out.download() - ref_out)) <= TOL * np.max(np.abs(ref_out))
    h.close()
    ctx.close()


@pytest.mark.gpu
def test_noalloc_rejects_problems_beyond_its_scratch():
    ctx = capi.Context(0)
    step = SiteStep.from_nac(os.path.join(GOLD, "heff_struct_cyl8x4_D1024.nac"))
    psi, L, R = step.synthetic_device(ctx, seed=3)
    out = capi.DeviceArray(ctx, step.psi_dim)
    rc = _noalloc(step, _blocks(step.L), _blocks(step.R), L, R, psi, out, False, ctx.stream)
    assert rc == -1  # DMRG_E_ARG, before any device work
    assert b"static scratch holds" in capi.lib().dmrg_last_error()
    ctx.close()


class _FakeDev:
    """A non-null stand-in for a device pointer: the validation under test
    rejects the call before any pointer is used or any CUDA call is made."""
    ptr = 0x1000


def test_noalloc_rejects_malformed_tables_on_the_host():
    """A ket block outside the sector range, a physics index outside [0, d) and
    an environment block outside its sector range each return DMRG_E_ARG before
    any device work, as dmrg_heff_create does (runs without a GPU)."""
    step = SiteStep.from_nac(os.path.join(GOLD, "heff_c158.nac"))
    Lb, Rb = _blocks(step.L), _blocks(step.R)
    dev = _FakeDev()
    site = step.site
    site.phys = site.phys.copy()  # writable copies of the tables to corrupt
    site.ket = capi.BlockSpec(site.ket.left.copy(), site.ket.right.copy(), site.ket.rows, site.ket.cols)
    good_phys = site.phys.copy()
    # a physics index >= d for the first ket block's sector pair
    k0 = (int(site.ket.left[0]), int(site.ket.right[0]))
    site.phys[k0[0] * site.nr + k0[1]] = site.d
    assert _noalloc(step, Lb, Rb, dev, dev, dev, dev, False, None) == -1
    assert b"physics index" in capi.lib().dmrg_last_error()
    site.phys[:] = good_phys
    # a ket block whose left sector is outside [0, nl)
    saved = int(site.ket.left[0])
    site.ket.left[0] = site.nl
    assert _noalloc(step, Lb, Rb, dev, dev, dev, dev, False, None) == -1
    assert b"ket block list" in capi.lib().dmrg_last_error()
    site.ket.left[0] = saved
    # an L block whose ket sector is negative
    bad = [capi.BlockSpec(s.left.copy(), s.right.copy(), s.rows, s.cols) for s in step.L]
    o = next(i for i, s in enumerate(bad) if len(s.left))
    bad[o].right[0] = -1
    assert _noalloc(step, _blocks(bad), Rb, dev, dev, dev, dev, False, None) == -1
    assert b"L[" in capi.lib().dmrg_last_error()
