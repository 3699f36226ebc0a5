"""a2/a3 parity: environment updates against the reference's outputs.
Block maps bit-exact; values within 1e-12 of the largest reference entry."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from dmrgcc_b200.problem import read_nac as pread
from oracle import dmrg_oracle as O
from oracle.nac import read_nac

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _spec(d, p):
    return capi.BlockSpec(d[p + ".left"], d[p + ".right"], d[p + ".rows"], d[p + ".cols"])


@pytest.mark.parametrize("call", [173, 187])
def test_env_update_matches_reference(ctx, call):
    d = pread(os.path.join(GOLD, f"env_c{call}.nac"))
    side = 0 if d["left"][0] else 1
    nl, nr = len(d["lattice.left_dim"]), len(d["lattice.right_dim"])
    dd, lb, rb = (int(x) for x in d["op.dims"])
    site = capi.SiteProblem(nl, nr, d["lattice.physics_index"], _spec(d, "lattice.ket"),
                            np.asarray(d["op.W"]).reshape(lb, rb, dd, dd))
    nin = int(d["env_in.bond"][0])
    specs = [_spec(d, f"env_in.{o}") for o in range(nin)]
    e = capi.Env(ctx, side, site, specs)
    nout = int(d["env_out.bond"][0])
    assert e.out_bond == nout
    for o, blk in enumerate(e.out_blocks()):
        assert np.array_equal(blk.left, d[f"env_out.{o}.left"])
        assert np.array_equal(blk.right, d[f"env_out.{o}.right"])
        assert np.array_equal(blk.rows, d[f"env_out.{o}.rows"])
        assert np.array_equal(blk.cols, d[f"env_out.{o}.cols"])
    ket = capi.DeviceArray.from_host(ctx, d["lattice.ket.data"])
    ein = capi.DeviceArray.from_host(ctx, np.concatenate([d[f"env_in.{o}.data"] for o in range(nin)]))
    eout = capi.DeviceArray(ctx, e.out_size)
    e.apply(ket, ein, eout)
    ctx.sync()
    got = eout.download()
    ref = np.concatenate([d[f"env_out.{o}.data"] for o in range(nout)])
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    alg, exe = e.flops()
    assert alg > 0 and exe > 0
