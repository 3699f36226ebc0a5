"""Two-site DMRG sweeps (dmrg_run_options_t.two_site) on the device.

The reference has no two-site mode (its sweep is single-site with subspace
expansion), so the two-site engine is validated against the reference's own
converged single-site results and against exact diagonalisation:

* 6-site chain and 3x3 cylinder: the final energy equals the exact ground-state
  energy (oracle/ed.py, which reproduces the reference's runs) to 1e-10 per
  site;
* 16-site chain (D=64): the final energy is at or below the reference's own
  single-site results at the same D (every gauge of gauge_spread_chain16.txt:
  the single-site sweep stops 1.7e-6 above the two-site one) and within 1e-10
  per site above the reference's converged D=256 energy
  (converged_chain16.txt), a variational bound up to its own convergence;
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
    with open(os.path.join(GOLD, "converged_chain16.txt")) as f:
        e256 = float([ln for ln in f if not ln.startswith("#")][-1])
    e = rec["energy"][-1]
    assert e <= min(ens.values()) + 1e-10 * 16, (e, min(ens.values()))
    assert -1e-10 <= (e - e256) / 16 <= 1e-10, (e, e256)
    assert np.all(np.diff(e_half[2:]) <= 1e-10 * 16)
