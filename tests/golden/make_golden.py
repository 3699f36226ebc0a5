"""Regenerates the golden fixtures in this directory from the reference itself.

Runs the unmodified reference DMRG, built from its own sources by oracle/Makefile
(`make -C oracle`), under the instrumented driver oracle/_ref/probe_dump with one
BLAS thread, on the 16-site Bose-Hubbard chain input (dmrgcc_b200/inputs/
chain16_spinless.in), and keeps:

  steps_chain16.txt     every Lanczos call: index, site, niter, psi_dim, energy
  heff_c<k>.nac         an H_eff*psi problem and the reference's output
  lanczos_c<k>.nac      the energy and ground vector LanczosMethod returned
  env_c<k>.nac          an environment update, inputs and outputs
  canon_c<k>.nac        a canonicalisation (SVD truncation), before and after
  steps_chain6.txt, steps_cylinder3x3.txt   whole runs of two small inputs
  trace_gauge_<input>.txt   whole runs of the three inputs with the free signs of
                        LAPACK's singular vectors / eigenvectors fixed by the
                        library's convention (PROBE_GAUGE=1): one line per
                        operation (E: Lanczos energy; X: expansion, C:
                        canonicalisation with its truncation gaps, T: match,
                        M: merge, with the sector dimensions after it)
  model_chain16.nac     the MPO per site and the quantum tables (first call)
  quicksort_cases.txt   inputs with ties and the index order the reference's
                        QuickSort (src/util/general.ih) returns (probe_sort)
  record_chain6.dat     the reference's checkpoint file (cache_record) of the
                        6-site chain after its first two sweeps, gauge-pinned
  trace_gauge_chain6_resume.txt, steps_chain6_resume.txt   the gauge-pinned
                        reference run resumed from that file (cache_resume,
                        full sweep table)

Usage: python tests/golden/make_golden.py [--cylinder] [--resume-only]
  --resume-only regenerates only the checkpoint fixtures.
  --cylinder additionally dumps the block structure (no values) of the 8x4
  cylinder at bond dimension 1024, site 16 (minutes of CPU), into
  heff_struct_cyl8x4_D1024.nac.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PROBE = os.path.join(ROOT, "oracle", "_ref", "probe_dump")
PROBE_SORT = os.path.join(ROOT, "oracle", "_ref", "probe_sort")

# Lanczos call k of the 16-site chain = half-sweep k // 15, k % 15-th site visited.
HEFF_CALLS = [20, 59, 158]  # psi_dim 181 (dense H_eff kept), 86 (dense ED branch), D=64 site 8
ENV_CALLS = [173, 187]   # left update site 8 (half-sweep 10), right update site 8 (11)
CANON_CALLS = [160, 174]  # expansion-on left/right canonicalisation at site 8, D=64


def run_probe(inp: str, out: str, env_extra: dict) -> None:
    env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1", PROBE_OUT=out, **env_extra)
    with open(os.path.join(out, "log.txt"), "w") as log:
        subprocess.run([PROBE, inp], env=env, stdout=log, stderr=subprocess.STDOUT, check=True, cwd=out)


def gauge_trace(name: str) -> None:
    """Structure trace of a gauge-pinned reference run (norm, rand-count and
    per-block fields dropped; they are diagnostics, not fixtures)."""
    t = tempfile.mkdtemp(prefix="golden_gauge_" + name)
    run_probe(os.path.join(ROOT, "dmrgcc_b200", "inputs", f"{name}_spinless.in"), t,
              {"PROBE_GAUGE": "1", "PROBE_TRACE": "1"})
    with open(os.path.join(t, "trace.txt")) as f, open(os.path.join(HERE, f"trace_gauge_{name}.txt"), "w") as g:
        for line in f:
            if line.startswith("Y"):
                continue
            parts = [p for p in line.split() if not p.startswith(("N:", "Q:", "S:"))]
            g.write(" ".join(parts) + "\n")


def final_energy(log_path: str) -> float:
    """The last `... energy = E` line the reference printed (real_tensor_rundmrg.cc:216)."""
    with open(log_path) as f:
        return [float(ln.split("=")[1]) for ln in f if "energy =" in ln][-1]


def gauge_spread(name: str, seeds, runs=None) -> None:
    """gauge_spread_<name>.txt: final energies of equally valid runs of the
    reference on one input (1 BLAS thread): `stock` (LAPACK's own signs),
    `pinned` (PROBE_GAUGE=1, the library's sign convention) and `seed s`
    (PROBE_GAUGE_SEED=s: every free sign of LAPACK's singular vectors and
    eigenvectors flipped at random).  Their spread is the reference's own
    run-to-run spread of the final energy under a choice the algorithm leaves
    free.  `runs` maps a label to an existing run directory (holding log.txt)
    to reuse instead of running it again."""
    runs = dict(runs or {})
    inp = os.path.join(ROOT, "dmrgcc_b200", "inputs", f"{name}_spinless.in")
    todo = [("stock", {}), ("pinned", {"PROBE_GAUGE": "1"})] + [(f"seed {s}", {"PROBE_GAUGE_SEED": str(s)})
                                                                 for s in seeds]
    rows = []
    for label, env in todo:
        d = runs.get(label)
        if d is None:
            d = tempfile.mkdtemp(prefix=f"golden_spread_{name}_")
            run_probe(inp, d, env)
        rows.append((label, final_energy(os.path.join(d, "log.txt"))))
    with open(os.path.join(HERE, f"gauge_spread_{name}.txt"), "w") as f:
        f.write(f"# final energy of the reference on {name}_spinless.in, 1 BLAS thread, per sign gauge\n")
        for label, e in rows:
            f.write(f"{label.replace(' ', '_')} {e:.12f}\n")


def input_with(src: str, **values) -> str:
    """The input file text `src` with the given `key = value` lines replaced."""
    import re

    for k, v in values.items():
        src, n = re.subn(rf"(?m)^(\s*){k}\s*=.*$", rf"\g<1>{k} = {v}", src)
        assert n == 1, k
    return src


def resume_case() -> None:
    """Checkpoint fixtures: the gauge-pinned reference records the 6-site chain
    after two sweeps (cache_record, RealTensorSpace::WriteTensorSpace), then a
    second reference run resumes from that file with the full sweep table
    (cache_resume, ReadTensorSpace)."""
    src = open(os.path.join(ROOT, "dmrgcc_b200", "inputs", "chain6_spinless.in")).read()
    t = tempfile.mkdtemp(prefix="golden_record_")
    rec_in = os.path.join(t, "record.in")
    with open(rec_in, "w") as f:
        f.write(input_with(src, num_sweep=2, cache_record="true", cache_name=t, record_name="record.dat"))
    run_probe(rec_in, t, {"PROBE_GAUGE": "1"})
    record = os.path.join(HERE, "record_chain6.dat")
    shutil.copy(os.path.join(t, "record.dat"), record)
    t2 = tempfile.mkdtemp(prefix="golden_resume_")
    res_in = os.path.join(t2, "resume.in")
    with open(res_in, "w") as f:
        f.write(input_with(src, cache_resume="true", resume_name=record))
    run_probe(res_in, t2, {"PROBE_GAUGE": "1", "PROBE_TRACE": "1"})
    shutil.copy(os.path.join(t2, "steps.txt"), os.path.join(HERE, "steps_chain6_resume.txt"))
    with open(os.path.join(t2, "trace.txt")) as f, \
            open(os.path.join(HERE, "trace_gauge_chain6_resume.txt"), "w") as g:
        for line in f:
            if line.startswith("Y"):
                continue
            parts = [p for p in line.split() if not p.startswith(("N:", "Q:", "S:"))]
            g.write(" ".join(parts) + "\n")


def quicksort_cases() -> None:
    import numpy as np

    rng = np.random.default_rng(7)
    lines = []
    for case in range(40):
        n = int(rng.integers(1, 60))
        flag = int(case % 2)
        pool = rng.choice([0.0, 0.125, 0.25, 0.5, 0.75, 1.0, 1e-13], size=int(rng.integers(1, 7)))
        vals = rng.choice(pool, size=n) if case % 3 else rng.random(n)
        lines.append(f"{n} {flag} " + " ".join(repr(float(v)) for v in vals))
    inp = "\n".join(lines) + "\n"
    r = subprocess.run([PROBE_SORT], input=inp, capture_output=True, text=True, check=True)
    outs = r.stdout.strip("\n").split("\n")
    with open(os.path.join(HERE, "quicksort_cases.txt"), "w") as f:
        for a, b in zip(lines, outs):
            f.write(a + "\n" + b + "\n")


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--cylinder", action="store_true")
    ap.add_argument("--resume-only", action="store_true")
    ap.add_argument("--spread", metavar="INPUT", help="only the gauge-spread fixture of one input "
                    "(chain16 or cylinder8x4; the cylinder takes about an hour per run)")
    ap.add_argument("--seeds", type=int, default=8, help="random-gauge runs for --spread")
    ap.add_argument("--reuse", action="append", default=[], metavar="LABEL=DIR",
                    help="for --spread: take run LABEL (stock, pinned, 'seed s') from DIR/log.txt")
    args = ap.parse_args()
    if not (os.path.exists(PROBE) and os.path.exists(PROBE_SORT)):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-j8"], check=True)
    if args.resume_only:
        resume_case()
        return 0
    if args.spread:
        gauge_spread(args.spread, range(1, args.seeds + 1), dict(r.split("=", 1) for r in args.reuse))
        return 0
    quicksort_cases()
    tmp = tempfile.mkdtemp(prefix="golden_")
    inp = os.path.join(ROOT, "dmrgcc_b200", "inputs", "chain16_spinless.in")
    run_probe(inp, tmp, {
        "PROBE_HEFF": ",".join(map(str, HEFF_CALLS)),
        "PROBE_ENV": ",".join(map(str, ENV_CALLS)),
        "PROBE_CANON": ",".join(map(str, CANON_CALLS)),
    })
    shutil.copy(os.path.join(tmp, "steps.txt"), os.path.join(HERE, "steps_chain16.txt"))
    shutil.copy(os.path.join(tmp, "model.nac"), os.path.join(HERE, "model_chain16.nac"))
    for name in ("chain6", "cylinder3x3"):
        t = tempfile.mkdtemp(prefix="golden_" + name)
        run_probe(os.path.join(ROOT, "dmrgcc_b200", "inputs", f"{name}_spinless.in"), t, {})
        shutil.copy(os.path.join(t, "steps.txt"), os.path.join(HERE, f"steps_{name}.txt"))
    for name in ("chain6", "cylinder3x3", "chain16"):
        gauge_trace(name)
    resume_case()
    for kind, calls in (("heff", HEFF_CALLS), ("lanczos", HEFF_CALLS), ("env", ENV_CALLS), ("canon", CANON_CALLS)):
        for c in calls:
            shutil.copy(os.path.join(tmp, f"{kind}_{c}.nac"), os.path.join(HERE, f"{kind}_c{c}.nac"))
    if args.cylinder:
        tmp2 = tempfile.mkdtemp(prefix="golden_cyl_")
        inp2 = os.path.join(ROOT, "dmrgcc_b200", "inputs", "cylinder8x4_spinless.in")
        # Lanczos call 388 = half-sweep 12 (first D=1024 sweep with noise off), site 16.
        env = {"PROBE_HEFF": "388", "PROBE_STRUCT_ONLY": "1", "PROBE_STOP": "388"}
        env2 = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count()), OPENBLAS_NUM_THREADS=str(os.cpu_count()),
                    PROBE_OUT=tmp2, **env)
        with open(os.path.join(tmp2, "log.txt"), "w") as log:
            subprocess.run([PROBE, inp2], env=env2, stdout=log, stderr=subprocess.STDOUT, check=True, cwd=tmp2)
        shutil.copy(os.path.join(tmp2, "heff_388.nac"), os.path.join(HERE, "heff_struct_cyl8x4_D1024.nac"))
        shutil.copy(os.path.join(tmp2, "steps.txt"), os.path.join(HERE, "steps_cyl8x4_to_D1024.txt"))
        shutil.copy(os.path.join(tmp2, "model.nac"), os.path.join(HERE, "model_cyl8x4.nac"))
    return 0


if __name__ == "__main__":
    sys.exit(main())
