"""The seeded 64-instance U/t scan workload (dmrgcc_b200/scan.py), host side:
the generator reproduces the instance list that the committed reference
energies (tests/golden/scan64_reference.txt) were computed on, and every input
file it writes is a valid input of the reference's format that the library's
model layer builds (MPO of the open chain with U_ref = U/2)."""
import os

import numpy as np

from dmrgcc_b200 import capi, scan

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _fixture():
    rows = []
    with open(os.path.join(GOLD, "scan64_reference.txt")) as f:
        for ln in f:
            if ln.startswith("#") or not ln.strip():
                continue
            i, L, U, e = ln.split()
            rows.append((int(i), int(L), float(U), float(e)))
    return rows


def test_generator_reproduces_the_reference_instances():
    rows = _fixture()
    insts = scan.instances()
    assert len(rows) == len(insts) == scan.N_INSTANCES
    for (i, L, U, e), inst in zip(rows, insts):
        assert inst["L"] == L and inst["L"] in scan.LENGTHS
        assert inst["U"] == U and 1.0 <= U <= 20.0
        # a chain of L sites at unit filling: the energy is negative and of order L
        assert -3.0 * L < e < 0.0


def test_every_scan_input_builds_its_model(tmp_path):
    paths = scan.write_inputs(str(tmp_path))
    assert len(paths) == scan.N_INSTANCES
    for p, inst in zip(paths, scan.instances()):
        m = capi.Model(p)
        assert (m.num_site, m.physics_dim) == (inst["L"], 4)
        # one MPO entry of a middle site is the on-site operator
        # diag(U_ref n (n - 1)), n = 0..3, with U_ref = U / 2 (mu = 0)
        W = m.mpo(inst["L"] // 2)
        diag = np.array([inst["U"] / 2.0 * n * (n - 1) for n in range(4)])
        hits = [np.allclose(np.diag(W[a, b]), diag, rtol=0, atol=1e-12) and
                np.count_nonzero(W[a, b] - np.diag(np.diag(W[a, b]))) == 0
                for a in range(W.shape[0]) for b in range(W.shape[1])]
        assert any(hits), p
        m.close()
