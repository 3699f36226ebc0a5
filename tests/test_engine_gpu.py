"""Whole DMRG runs on the device (the sweep engine) against the reference's own
runs of the same input files (tests/golden/steps_*.txt) and exact
diagonalisation.

Bookkeeping: psi_dim of every site step equals the reference's (the block maps
and every truncation decision agree).  Energies: each step within 1e-8 of the
reference's (both are converged Lanczos values of slightly different round-off
histories) and the final energy within 1e-10 per site."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from oracle.ed import ground_energy

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
INPUTS = os.path.join(ROOT, "dmrgcc_b200", "inputs")

CASES = [
    ("chain6_spinless.in", "steps_chain6.txt", 6, (6, 1, 6, 3, -1.0, 0.0, 2.0, 0.0, False, False)),
    ("cylinder3x3_spinless.in", "steps_cylinder3x3.txt", 9, (3, 3, 5, 3, -1.0, -1.0, 4.0, 0.0, False, True)),
    ("chain16_spinless.in", "steps_chain16.txt", 16, None),
]


@pytest.mark.parametrize("inp,steps,nsite,ed", CASES)
def test_engine_matches_reference_run(ctx, inp, steps, nsite, ed):
    ref = np.loadtxt(os.path.join(GOLD, steps))
    run = capi.Run(ctx, os.path.join(INPUTS, inp))
    run.execute()
    rec = run.steps()
    assert len(rec["energy"]) == len(ref)
    # site order of the sweep and the block structure at every step
    assert np.array_equal(rec["site"], ref[:, 1].astype(int))
    assert np.array_equal(rec["psi_dim"], ref[:, 3].astype(np.int64))
    assert np.max(np.abs(rec["energy"] - ref[:, 4])) <= 1e-8
    assert abs(rec["energy"][-1] - ref[-1, 4]) / nsite <= 1e-10
    e_half, t_half = run.half_sweeps()
    assert len(e_half) == len(ref) // (nsite - 1)
    assert np.all(rec["discarded"] >= 0)
    if ed is not None:
        assert abs(rec["energy"][-1] - ground_energy(*ed)) / nsite <= 1e-10
