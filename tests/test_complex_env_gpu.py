"""Complex environment updates on the device (dmrg_zenv_create / _apply)
against the reference's ComplexTensorContraction::Left/RightComputeTensorContraction
(the bra Hermitian-conjugated) on the Hofstadter fixtures: block maps
bit-exact, values within 1e-12 of the largest entry."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from dmrgcc_b200.problem import read_nac

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _spec(d, p):
    return capi.BlockSpec(d[p + ".left"], d[p + ".right"], d[p + ".rows"], d[p + ".cols"])


@pytest.mark.parametrize("call", [219, 241])
def test_complex_env_update_matches_reference(ctx, call):
    d = read_nac(os.path.join(GOLD, f"zenv_hof_c{call}.nac"))
    side = 0 if d["left"][0] else 1
    nl, nr = len(d["lattice.left_dim"]), len(d["lattice.right_dim"])
    dd, lb, rb = (int(x) for x in d["op.dims"])
    Wc = np.asarray(d["op.W"]).view(np.complex128).reshape(lb, rb, dd, dd)
    site = capi.SiteProblem(nl, nr, d["lattice.physics_index"], _spec(d, "lattice.ket"), Wc.real)
    nin, nout = int(d["env_in.bond"][0]), int(d["env_out.bond"][0])
    e = capi.Env(ctx, side, site, [_spec(d, f"env_in.{o}") for o in range(nin)], Wc=Wc)
    assert e.out_bond == nout
    for o, blk in enumerate(e.out_blocks()):
        for f in ("left", "right", "rows", "cols"):
            assert np.array_equal(getattr(blk, f), d[f"env_out.{o}.{f}"]), (o, f)
    ket = capi.DeviceArray.from_host(ctx, np.asarray(d["lattice.ket.data"]))
    ein = capi.DeviceArray.from_host(ctx, np.concatenate([np.asarray(d[f"env_in.{o}.data"]) for o in range(nin)]))
    eout = capi.DeviceArray(ctx, 2 * e.out_size)
    e.apply(ket, ein, eout)
    ctx.sync()
    got = eout.download().view(np.complex128)
    ref = np.concatenate([np.asarray(d[f"env_out.{o}.data"]) for o in range(nout)]).view(np.complex128)
    assert got.shape == ref.shape
    assert np.max(np.abs(ref.imag)) > 0.0
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
