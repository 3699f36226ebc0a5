"""Whole DMRG runs on the device (the sweep engine) against the reference's own
runs of the same input files, and exact diagonalisation.

The subspace expansion multiplies the site tensor by random matrices in the
basis the previous SVDs chose, so a run's trajectory depends on the free signs
of singular vectors and eigenvectors, which LAPACK leaves unspecified.  The
library fixes them by a convention (largest-magnitude component of each left
singular vector / eigenvector positive); tests/golden/trace_gauge_*.txt are
reference runs with LAPACK's outputs pinned to the same convention
(oracle/probe/probe_dump.cc, PROBE_GAUGE=1).  Against those:

* every operation (expansion X, canonicalisation C, match T, merge M) leaves
  the same sector dimensions, and every Lanczos call (E) sees the same psi_dim,
  up to the first truncation whose decision is ill-conditioned in the reference
  itself: the last kept and first dropped singular values closer than 1e-8 of
  the tensor norm, or a kept value less than four decades above canpre (its
  count then rests on digits of the state beyond the ~1e-8 accuracy of a
  converged Lanczos vector).  A run may
  part from the reference only there; after it the two follow equally valid
  paths and only the final energies are compared;
* energies of aligned Lanczos calls agree to 5e-9 per site (both are converged
  to ~1e-15 on operators that differ by round-off accumulated over the run);
* final energies agree with the pinned reference and with the stock reference
  run (tests/golden/steps_*.txt) to 1e-10 / 1e-9 per site, and with exact
  diagonalisation to 1e-10 per site where it is affordable;
* final energies lie inside the reference's own spread over equally valid sign
  gauges (tests/golden/gauge_spread_*.txt: the stock run, the pinned run and
  runs with random signs), widened by 1e-10 per site.  On the 16-site chain
  that spread is 5.7e-10 per site: the stock reference alone is not
  reproducible to 1e-10 per site under a change of sign gauge."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi
from oracle.ed import ground_energy

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
INPUTS = os.path.join(ROOT, "dmrgcc_b200", "inputs")

CASES = [
    ("chain6", 6, (6, 1, 6, 3, -1.0, 0.0, 2.0, 0.0, False, False)),
    ("cylinder3x3", 9, (3, 3, 5, 3, -1.0, -1.0, 4.0, 0.0, False, True)),
    ("chain16", 16, None),
]
GAP_CUT = 1e-8   # max_dim cut: (sigma_kept_last - sigma_dropped_first) / ||A||_F
GAP_PRE = 1e4    # canpre cut: smallest kept sigma / canpre


def parse_trace(path):
    """[(tag, key, energy, gaps)]: key = the structure fields of the line."""
    rows = []
    with open(path) as f:
        for line in f:
            p = line.split()
            if not p or p[0] in ("Y", "L"):  # expansion blocks, Lanczos timings: diagnostics
                continue
            if p[0] == "E":
                rows.append(("E", f"{p[2]} {p[3]}", float(p[4]), None))
                continue
            gaps = None
            for x in p:
                if x.startswith("G:"):
                    gaps = tuple(float(v) for v in x[2:].split(","))
            key = " ".join(x for x in p if not x.startswith(("N:", "Q:", "S:", "G:")))
            rows.append((p[0], key, None, gaps))
    return rows


def aligned_prefix(ref, got, etol):
    """Number of leading operations on which `got` follows `ref`; fails unless
    the first difference is a canonicalisation that is ill-conditioned in `ref`."""
    assert len(ref) == len(got)
    for i, (r, g) in enumerate(zip(ref, got)):
        assert r[0] == g[0], f"operation {i}: {r[0]} vs {g[0]}"
        if r[1] != g[1]:
            assert r[0] == "C" and r[3] is not None, f"operation {i}: {r[1]} vs {g[1]}"
            cut, pre = r[3]
            assert 0.0 <= cut < GAP_CUT or pre < GAP_PRE, (
                f"operation {i}: truncation differs at a well-conditioned cut (gaps {cut:.3e}, {pre:.3e}): "
                f"{r[1]} vs {g[1]}")
            return i
        if r[0] == "E":
            assert abs(r[2] - g[2]) <= etol, f"operation {i}: energy {g[2]!r} vs {r[2]!r}"
    return len(ref)


@pytest.mark.gpu
@pytest.mark.parametrize("name,nsite,ed", CASES)
def test_engine_follows_reference_run(ctx, tmp_path, name, nsite, ed):
    ref_trace = parse_trace(os.path.join(GOLD, f"trace_gauge_{name}.txt"))
    stock = np.loadtxt(os.path.join(GOLD, f"steps_{name}.txt"))
    trace = str(tmp_path / "trace.txt")
    os.environ["DMRG_TRACE"] = trace
    try:
        run = capi.Run(ctx, os.path.join(INPUTS, f"{name}_spinless.in"))
        run.execute()
    finally:
        del os.environ["DMRG_TRACE"]
    got = parse_trace(trace)
    n_aligned = aligned_prefix(ref_trace, got, 5e-9 * nsite)
    assert n_aligned >= min(len(ref_trace), 250)
    rec = run.steps()
    ref_e = [r[2] for r in ref_trace if r[0] == "E"]
    assert len(rec["energy"]) == len(ref_e) == len(stock)
    assert np.array_equal(rec["site"], stock[:, 1].astype(int))
    assert abs(rec["energy"][-1] - ref_e[-1]) / nsite <= 1e-10
    assert abs(rec["energy"][-1] - stock[-1, 4]) / nsite <= 1e-9
    e_half, _ = run.half_sweeps()
    assert len(e_half) == len(stock) // (nsite - 1)
    assert np.all(rec["discarded"] >= 0)
    if ed is not None:
        assert abs(rec["energy"][-1] - ground_energy(*ed)) / nsite <= 1e-10
    spread = os.path.join(GOLD, f"gauge_spread_{name}.txt")
    if os.path.exists(spread):
        assert_within_gauge_spread(rec["energy"][-1], spread, nsite)


def gauge_ensemble(path):
    """{label: final energy} of the reference's runs under different, equally
    valid sign gauges of its SVDs / eigensolves (tests/golden/make_golden.py
    --spread)."""
    out = {}
    with open(path) as f:
        for line in f:
            if line.strip() and not line.startswith("#"):
                label, e = line.split()
                out[label] = float(e)
    return out


def assert_within_gauge_spread(energy, path, nsite):
    """The final energy lies inside the reference's own spread over sign gauges
    (stock LAPACK signs, the pinned convention, random signs), widened by
    1e-10 per site.  This spread is the reference's run-to-run variation under
    a choice its algorithm leaves free; 1e-10 per site from the stock run alone
    is a tighter bar than the reference meets against itself on these
    schedules."""
    ens = gauge_ensemble(path)
    lo, hi = min(ens.values()), max(ens.values())
    tol = 1e-10 * nsite
    assert lo - tol <= energy <= hi + tol, (energy, lo, hi)
    return lo, hi


def test_trace_comparison_rejects_a_well_conditioned_divergence():
    """The alignment check itself: a planted dimension change at a
    canonicalisation with a wide gap must fail; at a narrow gap it must pass."""
    ref = [("E", "0 P:3", -1.0, None), ("C", "C 0 0 L:1, R:2,", None, (1e-3, 1e9)),
           ("E", "1 P:9", -2.0, None)]
    got = [("E", "0 P:3", -1.0, None), ("C", "C 0 0 L:1, R:3,", None, None), ("E", "1 P:12", -2.1, None)]
    with pytest.raises(AssertionError):
        aligned_prefix(ref, got, 1e-9)
    narrow = [ref[0], ("C", "C 0 0 L:1, R:2,", None, (1e-12, 1e9)), ref[2]]
    assert aligned_prefix(narrow, got, 1e-9) == 1


def test_gauge_spread_check_rejects_an_energy_outside_it(tmp_path):
    """The spread check itself: an energy 1e-9 per site below the ensemble
    fails, one inside it passes (no GPU)."""
    p = tmp_path / "spread.txt"
    p.write_text("# test\nstock -10.0\npinned -10.000000001\nseed_1 -10.0000000005\n")
    assert_within_gauge_spread(-10.0000000007, str(p), 10)
    with pytest.raises(AssertionError):
        assert_within_gauge_spread(-10.000000001 - 1e-8, str(p), 10)


@pytest.mark.gpu
def test_cylinder8x4_D1024_final_energy_within_reference_spread(ctx):
    """The 8x4 cylinder (D 128 -> 1024, 8 sweeps) end to end on the device:
    the final energy lies within the reference's own gauge spread (stock,
    pinned and random-sign runs of the reference on the same input), widened by
    1e-10 per site, and the sites visited match the stock run's."""
    spread = os.path.join(GOLD, "gauge_spread_cylinder8x4.txt")
    if not os.path.exists(spread):
        pytest.skip("gauge_spread_cylinder8x4.txt not generated")
    run = capi.Run(ctx, os.path.join(INPUTS, "cylinder8x4_spinless.in"))
    run.execute()
    rec = run.steps()
    assert len(rec["energy"]) == 16 * 31
    assert np.all(rec["discarded"] >= 0)
    assert_within_gauge_spread(rec["energy"][-1], spread, 32)


@pytest.mark.gpu
@pytest.mark.parametrize("two_site", [False, True])
def test_spinful_run_matches_reference_and_ed(ctx, two_site):
    """The spinful U(1) x U(1) model end to end on the device (single-site with
    expansion, and two-site): the final energy equals the reference's converged
    run and exact diagonalisation to 1e-10 per MPS site."""
    from oracle.ed import ground_energy_spinful

    run = capi.Run(ctx, os.path.join(INPUTS, "spinful3x2.in"), model="real_spinful_bose_square", two_site=two_site)
    run.execute()
    e = run.steps()["energy"][-1]
    with open(os.path.join(GOLD, "spinful_reference.txt")) as f:
        e_ref = float([ln.split()[1] for ln in f if ln.startswith("spinful3x2")][0])
    assert abs(e - e_ref) / 12 <= 1e-10
    assert abs(e - ground_energy_spinful(3, 2, 3, 3, 3, -1.0, -1.0, 6.0, 6.0, 3.0, 0.0)) / 12 <= 1e-10
