"""Whole complex DMRG runs (ComplexTensorRundmrg): the Hofstadter model
(complex_spinful_bose_square, flux 1/6 on a 4x3 lattice periodic in y, 3
bosons of one species; every tensor complex: H_eff*psi, conjugated Lanczos,
environments, the real-form SVD, expansion and merge).

* the final energy equals exact diagonalisation with the Peierls phase
  (oracle/ed.py, pinned to the reference's own converged run) and the
  reference's final energy, to 1e-10 per lattice site;
* every half-sweep's energy after the first sweep is non-increasing;
* the same model without flux on the real path gives the same energy as the
  complex path run on it (one model, two fields)."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from oracle.ed import ground_energy_spinful

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
INPUT = os.path.join(ROOT, "dmrgcc_b200", "inputs", "hofstadter4x3.in")


def test_hofstadter_complex_run_matches_exact_diagonalisation(ctx):
    run = capi.Run(ctx, INPUT, model="complex_spinful_bose_square")
    run.execute()
    e_half, _ = run.half_sweeps()
    e_ed = ground_energy_spinful(4, 3, 3, 0, 3, -1.0, -1.0, 10.0, 0.0, 0.0, 0.0, False, True,
                                 flux=0.16666666666666666)
    with open(os.path.join(GOLD, "steps_hofstadter4x3.txt")) as f:
        e_ref = float([ln.split() for ln in f if ln.strip() and not ln.startswith("#")][-1][4])
    assert abs(e_half[-1] - e_ed) / 12 <= 1e-10, (e_half[-1], e_ed)
    assert abs(e_half[-1] - e_ref) / 12 <= 1e-10, (e_half[-1], e_ref)
    assert np.all(np.diff(e_half[2:]) <= 1e-10 * 12)


def test_complex_path_on_a_real_model_matches_the_real_path(ctx, tmp_path):
    src = open(INPUT).read().replace("flux = 0.16666666666666666", "flux = 0.0")
    p = tmp_path / "noflux.in"
    p.write_text(src)
    ez = capi.Run(ctx, str(p), model="complex_spinful_bose_square")
    ez.execute()
    er = capi.Run(ctx, str(p), model="real_spinful_bose_square")
    er.execute()
    e_ed = ground_energy_spinful(4, 3, 3, 0, 3, -1.0, -1.0, 10.0, 0.0, 0.0, 0.0, False, True)
    assert abs(ez.half_sweeps()[0][-1] - e_ed) / 12 <= 1e-10
    assert abs(er.half_sweeps()[0][-1] - e_ed) / 12 <= 1e-10


def test_hofstadter_6x6_matches_the_reference_run(ctx):
    """The 6x6 Hofstadter geometry (periodic in y, flux
    1/6, 4 bosons, D <= 256; hofstadter6x6.in): the final energy within 1e-10
    per lattice site of the reference's run of the same input
    (tests/golden/hofstadter6x6_reference.txt)."""
    run = capi.Run(ctx, os.path.join(ROOT, "dmrgcc_b200", "inputs", "hofstadter6x6.in"),
                   model="complex_spinful_bose_square")
    run.execute()
    with open(os.path.join(GOLD, "hofstadter6x6_reference.txt")) as f:
        e_ref = float([ln.split()[1] for ln in f if ln.startswith("hofstadter6x6")][0])
    e = run.half_sweeps()[0][-1]
    assert abs(e - e_ref) / 36 <= 1e-10, (e, e_ref)
