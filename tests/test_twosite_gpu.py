"""Two-site DMRG sweeps (dmrg_run_options_t.two_site) on the device.

The reference has no two-site mode (its sweep is single-site with subspace
expansion), so the two-site engine is validated against the reference's own
converged single-site results and against exact diagonalisation:

* 6-site chain and 3x3 cylinder: the final energy equals the exact ground-state
  energy (oracle/ed.py, which reproduces the reference's runs) to 1e-10 per
  site;
* 16-site chain (D=64): the final energy lies within the reference's own
  gauge spread of the single-site run's final energy (gauge_spread_chain16.txt),
  widened by 1e-9 per site (two different algorithms on the same D);
* every half-sweep's energy is non-increasing after the first full sweep
  (variational at fixed D), the discarded weights are non-negative, and the
  Krylov dimensions stay within niter."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from oracle.ed import ground_energy

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
INPUTS = os.path.join(ROOT, "dmrgcc_b200", "inputs")

pytestmark = pytest.mark.gpu


def _run(ctx, name, **kw):
    run = capi.Run(ctx, os.path.join(INPUTS, f"{name}_spinless.in"), two_site=True, **kw)
    run.execute()
    return run


@pytest.mark.parametrize("name,nsite,ed", [
    ("chain6", 6, (6, 1, 6, 3, -1.0, 0.0, 2.0, 0.0, False, False)),
    ("cylinder3x3", 9, (3, 3, 5, 3, -1.0, -1.0, 4.0, 0.0, False, True)),
])
def test_twosite_matches_exact_diagonalisation(ctx, name, nsite, ed):
    run = _run(ctx, name)
    rec = run.steps()
    e_half, _ = run.half_sweeps()
    assert abs(rec["energy"][-1] - ground_energy(*ed)) / nsite <= 1e-10
    assert np.all(rec["discarded"] >= 0)
    assert np.all(rec["lanczos_dim"] >= 0) and np.all(rec["lanczos_dim"] <= 100)
    assert np.all(np.diff(e_half[2:]) <= 1e-10 * nsite)
    # one record per bond and half-sweep
    assert len(rec["energy"]) == len(e_half) * (nsite - 1)


def test_twosite_chain16_matches_the_single_site_reference(ctx):
    from test_engine_gpu import gauge_ensemble

    run = _run(ctx, "chain16")
    rec = run.steps()
    e_half, _ = run.half_sweeps()
    ens = gauge_ensemble(os.path.join(GOLD, "gauge_spread_chain16.txt"))
    lo, hi = min(ens.values()), max(ens.values())
    e = rec["energy"][-1]
    assert lo - 1e-9 * 16 <= e <= hi + 1e-9 * 16, (e, lo, hi)
    assert np.all(np.diff(e_half[2:]) <= 1e-10 * 16)
