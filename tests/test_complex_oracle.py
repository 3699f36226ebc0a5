"""The complex path's oracle pinned to the reference (CPU): the numpy restatement
of MultiplyEffectHamilton (oracle/dmrg_oracle.py) run on complex blocks
reproduces the reference's complex H_eff*psi (ComplexTensorContraction::
MultiplyEffectHamilton, src/dmrg/complexdmrg/complex_tensor_contraction.cc:
1244-1312) on the Bose-Hubbard-Hofstadter fixtures of
tests/golden/make_golden.py --complex, and the complex H_eff is Hermitian."""
import os

import numpy as np
import pytest

from oracle import dmrg_oracle as O
from oracle.nac import read_nac

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def zblocks(d, p):
    """A complex block list from interleaved (re, im) data."""
    left = [int(x) for x in d[p + ".left"]]
    right = [int(x) for x in d[p + ".right"]]
    rows, cols = d[p + ".rows"], d[p + ".cols"]
    data = np.asarray(d[p + ".data"]).view(np.complex128)
    mats, pos = [], 0
    for r, c in zip(rows, cols):
        mats.append(data[pos:pos + r * c].reshape(r, c).copy())
        pos += r * c
    return O.BlockList(left, right, mats)


def zproblem(d):
    nl, nr = len(d["lattice.left_dim"]), len(d["lattice.right_dim"])
    lat = O.Lattice(physics_dim=int(d["lattice.physics_dim"][0]), left_block=list(range(nl)),
                    left_dim=[int(x) for x in d["lattice.left_dim"]], right_block=list(range(nr)),
                    right_dim=[int(x) for x in d["lattice.right_dim"]],
                    physics_index=np.asarray(d["lattice.physics_index"]).reshape(nl, nr),
                    ket=zblocks(d, "lattice.ket"))
    dd, lb, rb = (int(x) for x in d["op.dims"])
    W = np.asarray(d["op.W"]).view(np.complex128).reshape(lb, rb, dd, dd)
    L = [zblocks(d, f"L.{o}") for o in range(lb)]
    R = [zblocks(d, f"R.{o}") for o in range(rb)]
    return lat, W, L, R


@pytest.mark.parametrize("call", [182, 196])
def test_oracle_complex_heff_matches_reference(call):
    d = read_nac(os.path.join(GOLD, f"zheff_hof_c{call}.nac"))
    lat, W, L, R = zproblem(d)
    out = np.zeros(lat.psi_dim(), dtype=np.complex128)
    O.multiply_effect_hamilton(lat, W, L, R, out)
    ref = np.asarray(d["heff_out"]).view(np.complex128)
    assert np.max(np.abs(ref.imag)) > 1e-3 * np.max(np.abs(ref))  # genuinely complex
    assert np.max(np.abs(out - ref)) <= 1e-13 * np.max(np.abs(ref))


def test_complex_heff_is_hermitian():
    d = read_nac(os.path.join(GOLD, "zheff_hof_c182.nac"))
    lat, W, L, R = zproblem(d)
    n = lat.psi_dim()
    H = np.zeros((n, n), dtype=np.complex128)
    for c in range(n):
        e = np.zeros(n, dtype=np.complex128)
        e[c] = 1.0
        lat.ket.unvectorize(e)
        col = np.zeros(n, dtype=np.complex128)
        O.multiply_effect_hamilton(lat, W, L, R, col)
        H[:, c] = col
    assert np.max(np.abs(H - H.conj().T)) <= 1e-12 * np.max(np.abs(H))
    ref = read_nac(os.path.join(GOLD, "zlanczos_hof_c182.nac"))
    assert abs(np.linalg.eigvalsh(H)[0] - float(ref["energy"][0])) <= 1e-12 * 24
