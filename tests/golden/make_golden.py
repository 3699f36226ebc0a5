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


# D=1024 fixtures of the 8x4 cylinder, half-sweeps 8 (left to right) and 9 (right
# to left), both with expansion on: (kind, probe call, extra probe settings,
# Lanczos call to stop after).  Env call = 31 + 31 h + k, canonicalisation call
# = 64 + 31 h + k, Lanczos call = 31 h + k for step k of half-sweep h.
D1024_CASES = [
    ("env", 283, {"PROBE_ENV": "283", "PROBE_SYNTH": "11"}, 253),     # left update, site 4
    ("env", 314, {"PROBE_ENV": "314", "PROBE_SYNTH": "12"}, 284),     # right update, site 27
    ("canon", 318, {"PROBE_CANON": "318", "PROBE_SYNTH": "13"}, 255),  # left, site 6, expanded
    ("canon", 349, {"PROBE_CANON": "349", "PROBE_SYNTH": "14"}, 286),  # right, site 25, expanded
    ("lanczos", 252, {"PROBE_HEFF": "252", "PROBE_ROUND_F32": "1"}, 252),  # site 4
]
N_SAMPLES = 4096


def _structure(d: dict, prefixes) -> dict:
    """The block-structure arrays of a dump (no values)."""
    return {k: v for k, v in d.items()
            if any(k.startswith(p) for p in prefixes) and not k.endswith(".data")}


def _samples(values, seed: int):
    """Seeded sample positions (with the first and last element) and the values there."""
    import numpy as np

    n = len(values)
    idx = np.unique(np.concatenate([[0, n - 1], np.random.default_rng(seed).integers(0, n, N_SAMPLES)]))
    return idx.astype(np.int32), np.asarray(values)[idx]


def d1024_fixture(kind: str, call: int, run_dir: str) -> None:
    """Compact fixture from a reference dump at D=1024 (the dump itself is tens of MB):
    env / canon: the dump's block structures, the seed of its synthetic inputs
      (PROBE_SYNTH: ket values, then the incoming environment, from the splitmix64
      stream) and a digest of the reference's output: seeded sample entries, the
      sum of squares per MPO bond (env) or the singular values and the sampled
      gauge-invariant products U S V^T per block (canon);
    lanczos: the float32-rounded environments and start vector it ran on
      (PROBE_ROUND_F32), the energy and the ground vector (float32)."""
    import numpy as np

    sys.path.insert(0, ROOT)
    from oracle.nac import read_nac, write_nac

    if kind == "env":
        d = read_nac(os.path.join(run_dir, f"env_{call}.nac"))
        out = _structure(d, ("left", "site", "synth_seed", "lattice.", "op.", "env_in.", "env_out."))
        bond = int(d["env_out.bond"][0])
        data = [np.asarray(d[f"env_out.{o}.data"]) for o in range(bond)]
        flat = np.concatenate(data) if data else np.zeros(0)
        out["digest.sumsq"] = np.array([float(np.sum(x * x)) for x in data])
        out["digest.index"], out["digest.value"] = _samples(flat, call)
        write_nac(os.path.join(HERE, f"env_cyl8x4_D1024_c{call}.nac"), out)
    elif kind == "canon":
        d = read_nac(os.path.join(run_dir, f"canon_{call}.nac"))
        left = bool(d["left"][0])
        out = _structure(d, ("left", "site", "synth_seed", "max_dim", "canpre", "before.", "after."))
        # singular values: row norms of S V^T (left) / column norms of U S (right)
        cr, cc = d["after.canonical.rows"], d["after.canonical.cols"]
        cdat = np.asarray(d["after.canonical.data"])
        kr, kc, kl, kri = d["after.ket.rows"], d["after.ket.cols"], d["after.ket.left"], d["after.ket.right"]
        kdat = np.asarray(d["after.ket.data"])
        coff = np.concatenate([[0], np.cumsum(cr.astype(np.int64) * cc)])
        koff = np.concatenate([[0], np.cumsum(kr.astype(np.int64) * kc)])
        sig, prods = [], []
        for s in range(len(cr)):
            c = cdat[coff[s]:coff[s + 1]].reshape(cr[s], cc[s])
            sig.append(np.linalg.norm(c, axis=1) if left else np.linalg.norm(c, axis=0))
        for k in range(len(kr)):
            b = kdat[koff[k]:koff[k + 1]].reshape(kr[k], kc[k])
            s = kri[k] if left else kl[k]
            c = cdat[coff[s]:coff[s + 1]].reshape(cr[s], cc[s])
            prods.append((b @ c if left else c @ b).ravel())
        out["digest.sigma_count"] = np.array([len(x) for x in sig], dtype=np.int32)
        out["digest.sigma"] = np.concatenate(sig)
        flat = np.concatenate(prods) if prods else np.zeros(0)
        out["digest.index"], out["digest.value"] = _samples(flat, call)
        out["digest.prod_sumsq"] = np.array([float(np.sum(flat * flat))])
        write_nac(os.path.join(HERE, f"canon_cyl8x4_D1024_c{call}.nac"), out)
    else:
        h = read_nac(os.path.join(run_dir, f"heff_{call}.nac"))
        lz = read_nac(os.path.join(run_dir, f"lanczos_{call}.nac"))
        arrays = {k: v for k, v in h.items() if not k.endswith(".data") and k != "heff_out" and k != "heff_dense"}
        for k, v in h.items():
            if k.endswith(".data"):
                f32 = np.asarray(v, dtype=np.float32)
                assert np.array_equal(f32.astype(np.float64), v), k  # the probe rounded them
                arrays[k] = f32
        arrays["energy"] = np.asarray(lz["energy"])
        arrays["ground"] = np.asarray(lz["lattice.ket.data"], dtype=np.float32)
        np.savez_compressed(os.path.join(HERE, f"lanczos_cyl8x4_D1024_c{call}.npz"), **arrays)


def d1024_fixtures(reuse: dict) -> None:
    """Runs the reference (1 BLAS thread) up to each D=1024 case, or reuses a
    finished run directory (label = the case's kind and call, e.g. 'env 283')."""
    inp = os.path.join(ROOT, "dmrgcc_b200", "inputs", "cylinder8x4_spinless.in")
    for kind, call, env, stop in D1024_CASES:
        d = reuse.get(f"{kind} {call}")
        if d is None:
            d = tempfile.mkdtemp(prefix=f"golden_d1024_{kind}_{call}_")
            run_probe(inp, d, dict(env, PROBE_STOP=str(stop)))
        d1024_fixture(kind, call, d)


def scan_reference(jobs: int) -> None:
    """scan64_reference.txt: the stock reference's final energy on each of the
    64 U/t-scan inputs (dmrgcc_b200/scan.py), 1 BLAS thread per process."""
    from concurrent.futures import ThreadPoolExecutor

    sys.path.insert(0, ROOT)
    from dmrgcc_b200 import scan

    tmp = tempfile.mkdtemp(prefix="golden_scan_")
    paths = scan.write_inputs(tmp)
    model = os.path.join(ROOT, "oracle", "_ref", "real_spinless_bose_square_model")
    env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1")

    def one(p):
        r = subprocess.run([model, p], capture_output=True, text=True, env=env, cwd=tmp, check=True)
        return [float(ln.split("=")[1]) for ln in r.stdout.splitlines() if "energy =" in ln][-1]

    with ThreadPoolExecutor(max_workers=jobs) as ex:
        energies = list(ex.map(one, paths))
    with open(os.path.join(HERE, "scan64_reference.txt"), "w") as f:
        f.write("# instance L U/t final energy of the stock reference (1 BLAS thread)\n")
        for i, (inst, e) in enumerate(zip(scan.instances(), energies)):
            f.write(f"{i} {inst['L']} {inst['U']:.17g} {e:.12f}\n")


def converged_reference() -> None:
    """converged_chain16.txt: the stock reference on chain16_spinless.in with its
    D ramp continued to 256 and six noiseless D=256 half-sweep pairs, a
    converged estimate of the ground-state energy (a variational bound for every
    run of the same model at D <= 256 up to its own convergence)."""
    src = open(os.path.join(ROOT, "dmrgcc_b200", "inputs", "chain16_spinless.in")).read()
    head, _ = src.split("maxm  maxb  niter  canpre  noise")
    rows = ([(16, 4)] * 2 + [(32, 5)] * 2 + [(64, 6)] * 2 + [(128, 7)] * 2 + [(256, 8)] * 2 + [(256, -1)] * 6)
    head = head.replace("num_sweep = 6", f"num_sweep = {len(rows) // 2}")
    text = head + "maxm  maxb  niter  canpre  noise\n" + "\n".join(
        f"        {m:<5d} 100   100    1E-12   {z}" for m, z in rows) + "\n    }\n}\n"
    tmp = tempfile.mkdtemp(prefix="golden_conv_")
    inp = os.path.join(tmp, "chain16_D256.in")
    with open(inp, "w") as f:
        f.write(text)
    model = os.path.join(ROOT, "oracle", "_ref", "real_spinless_bose_square_model")
    env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1")
    r = subprocess.run([model, inp], capture_output=True, text=True, env=env, cwd=tmp, check=True)
    e = [float(ln.split("=")[1]) for ln in r.stdout.splitlines() if "energy =" in ln]
    with open(os.path.join(HERE, "converged_chain16.txt"), "w") as f:
        f.write("# chain16_spinless.in with the D ramp continued to 256 (16->32->64->128->256, then 6 noiseless\n"
                "# D=256 sweeps), stock reference, 1 BLAS thread: energies of the last two half-sweeps\n")
        f.write(f"{e[-2]:.12f}\n{e[-1]:.12f}\n")


def complex_run_reference() -> None:
    """hofstadter6x6_reference.txt: the reference's final energy on
    hofstadter6x6.in (complex_spinful_bose_square_model, 1 BLAS thread): the
    6x6 Hofstadter geometry (flux 1/6, periodic in y) with 4 bosons (the reference's model
    crashes on this lattice with 5 or 6 bosons)."""
    tmp = tempfile.mkdtemp(prefix="golden_h66_")
    env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1")
    model = os.path.join(ROOT, "oracle", "_ref", "complex_spinful_bose_square_model")
    r = subprocess.run([model, os.path.join(ROOT, "dmrgcc_b200", "inputs", "hofstadter6x6.in")], capture_output=True,
                       text=True, env=env, cwd=tmp, check=True)
    e = [float(ln.split("=")[1]) for ln in r.stdout.splitlines() if "energy =" in ln][-1]
    with open(os.path.join(HERE, "hofstadter6x6_reference.txt"), "w") as f:
        f.write("# final energy of complex_spinful_bose_square_model on hofstadter6x6.in (1 BLAS thread)\n")
        f.write(f"hofstadter6x6 {e:.14f}\n")


SPINFUL_MODELS = ("spinful4x4", "spinful3x3_periodic_y")
COMPLEX_MODELS = ("hofstadter4x3",)


MERGE_CALLS = (38, 50)  # a left and a right merge (site 9, second sweep) of the 16-site chain run


def merge_fixtures() -> None:
    """merge_c<i>.nac: the inputs and output of the reference's
    Left/RightMergeTensorLattice at merge calls MERGE_CALLS of the 16-site chain
    run (1 BLAS thread): the site merged into, before and after, and the
    lattice whose canonical tensor is multiplied in."""
    tmp = tempfile.mkdtemp(prefix="golden_merge_")
    run_probe(os.path.join(ROOT, "dmrgcc_b200", "inputs", "chain16_spinless.in"), tmp,
              {"PROBE_MERGE": ",".join(map(str, MERGE_CALLS))})
    for c in MERGE_CALLS:
        shutil.copy(os.path.join(tmp, f"merge_{c}.nac"), os.path.join(HERE, f"merge_c{c}.nac"))


COMPLEX_SPINLESS_MODELS = ("chain16_spinless", "cylinder3x3_spinless")


def complex_spinless_fixtures() -> None:
    """model_complex_<input>.nac: the MPO (real and imaginary parts) and the
    quantum tables of the reference's complex spinless model
    (ComplexSpinlessBoseSquareSpace / ComplexSpinlessBoseSquareHamiltonian,
    oracle/_ref/probe_model ... spinless) on the spinless inputs."""
    sys.path.insert(0, ROOT)
    from oracle.nac import read_nac, write_nac

    probe = os.path.join(ROOT, "oracle", "_ref", "probe_model")
    for name in COMPLEX_SPINLESS_MODELS:
        tmp = tempfile.mkdtemp(prefix="golden_zmodel_")
        out = os.path.join(tmp, "model.nac")
        subprocess.run([probe, os.path.join(ROOT, "dmrgcc_b200", "inputs", f"{name}.in"), out, "spinless"],
                       check=True, stdout=subprocess.DEVNULL)
        write_nac(os.path.join(HERE, f"model_complex_{name}.nac"), read_nac(out))


def spinful_fixtures() -> None:
    """model_<input>.nac: the reference's spinful MPO and quantum tables
    (oracle/_ref/probe_model; the imaginary parts, zero at flux 0, are checked
    and dropped; kept for the Hofstadter input, whose flux makes them nonzero),
    and spinful_reference.txt: the reference's final energy on
    spinful3x2.in (complex_spinful_bose_square_model, 1 BLAS thread)."""
    import numpy as np

    sys.path.insert(0, ROOT)
    from oracle.nac import read_nac, write_nac

    probe = os.path.join(ROOT, "oracle", "_ref", "probe_model")
    for name in SPINFUL_MODELS:
        tmp = tempfile.mkdtemp(prefix="golden_model_")
        out = os.path.join(tmp, "model.nac")
        subprocess.run([probe, os.path.join(ROOT, "dmrgcc_b200", "inputs", f"{name}.in"), out], check=True,
                       stdout=subprocess.DEVNULL)
        d = read_nac(out)
        for k in [k for k in d if k.endswith(".Wi")]:
            assert not np.any(d[k]), k
            del d[k]
        write_nac(os.path.join(HERE, f"model_{name}.nac"), d)
    for name in COMPLEX_MODELS:  # Peierls phases: the imaginary parts are kept
        tmp = tempfile.mkdtemp(prefix="golden_model_")
        out = os.path.join(tmp, "model.nac")
        subprocess.run([probe, os.path.join(ROOT, "dmrgcc_b200", "inputs", f"{name}.in"), out], check=True,
                       stdout=subprocess.DEVNULL)
        write_nac(os.path.join(HERE, f"model_{name}.nac"), read_nac(out))
    tmp = tempfile.mkdtemp(prefix="golden_spinful_")
    env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1")
    model = os.path.join(ROOT, "oracle", "_ref", "complex_spinful_bose_square_model")
    r = subprocess.run([model, os.path.join(ROOT, "dmrgcc_b200", "inputs", "spinful3x2.in")], capture_output=True,
                       text=True, env=env, cwd=tmp, check=True)
    e = [float(ln.split("=")[1]) for ln in r.stdout.splitlines() if "energy =" in ln][-1]
    with open(os.path.join(HERE, "spinful_reference.txt"), "w") as f:
        f.write("# final energy of complex_spinful_bose_square_model on spinful3x2.in (1 BLAS thread)\n")
        f.write(f"spinful3x2 {e:.14f}\n")


ZHEFF_CALLS = [182, 196]  # site 2 (psi_dim 54: dense branch), site 12 (psi_dim 313), half-sweep 8
ZENV_CALLS = [219, 241]   # left update at site 12 (half-sweep 8), right update at site 12 (half-sweep 9)
ZCANON_CALLS = [244, 266]  # expanded left / right canonicalisation at site 12 (half-sweeps 8 / 9)


def complex_fixtures() -> None:
    """The complex path's fixtures: the reference's complex DMRG (spinful model
    executable with Ndown = 0 and flux 1/6: Bose-Hubbard-Hofstadter on a 4x3
    cylinder, dmrgcc_b200/inputs/hofstadter4x3.in) under oracle/_ref/probe_zdump,
    1 BLAS thread: zheff_hof_c<k>.nac / zlanczos_hof_c<k>.nac (an H_eff problem,
    the reference's H*psi on its ket, and LanczosMethod's energy and vector),
    zenv_hof_c<k>.nac (environment updates), steps_hofstadter4x3.txt."""
    tmp = tempfile.mkdtemp(prefix="golden_complex_")
    probe = os.path.join(ROOT, "oracle", "_ref", "probe_zdump")
    env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1", PROBE_OUT=tmp,
               PROBE_HEFF=",".join(map(str, ZHEFF_CALLS)), PROBE_ENV=",".join(map(str, ZENV_CALLS)),
               PROBE_CANON=",".join(map(str, ZCANON_CALLS)))
    with open(os.path.join(tmp, "log.txt"), "w") as log:
        subprocess.run([probe, os.path.join(ROOT, "dmrgcc_b200", "inputs", "hofstadter4x3.in")], env=env,
                       stdout=log, stderr=subprocess.STDOUT, check=True, cwd=tmp)
    for c in ZHEFF_CALLS:
        shutil.copy(os.path.join(tmp, f"zheff_{c}.nac"), os.path.join(HERE, f"zheff_hof_c{c}.nac"))
        shutil.copy(os.path.join(tmp, f"zlanczos_{c}.nac"), os.path.join(HERE, f"zlanczos_hof_c{c}.nac"))
    for c in ZENV_CALLS:
        shutil.copy(os.path.join(tmp, f"zenv_{c}.nac"), os.path.join(HERE, f"zenv_hof_c{c}.nac"))
    for c in ZCANON_CALLS:
        shutil.copy(os.path.join(tmp, f"zcanon_{c}.nac"), os.path.join(HERE, f"zcanon_hof_c{c}.nac"))
    shutil.copy(os.path.join(tmp, "steps.txt"), os.path.join(HERE, "steps_hofstadter4x3.txt"))


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
    ap.add_argument("--d1024", action="store_true", help="only the 8x4 cylinder D=1024 fixtures (each case "
                    "runs the reference up to its call: minutes of CPU)")
    ap.add_argument("--scan", action="store_true", help="only the 64-instance U/t scan reference energies")
    ap.add_argument("--spinful", action="store_true", help="only the spinful model fixtures")
    ap.add_argument("--complex-spinless", action="store_true", help="only the complex spinless model fixtures")
    ap.add_argument("--merge", action="store_true", help="only the merge fixtures of the 16-site chain")
    ap.add_argument("--complex", action="store_true", help="only the complex-path (Hofstadter) fixtures")
    ap.add_argument("--converged", action="store_true", help="only the converged chain16 energy (D=256)")
    ap.add_argument("--complex-run", action="store_true", help="only the reference energy of hofstadter6x6.in")
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
    if args.d1024:
        d1024_fixtures(dict(r.split("=", 1) for r in args.reuse))
        return 0
    if args.scan:
        scan_reference(os.cpu_count() or 4)
        return 0
    if args.spinful:
        spinful_fixtures()
        return 0
    if args.complex_spinless:
        complex_spinless_fixtures()
        return 0
    if args.merge:
        merge_fixtures()
        return 0
    if args.complex:
        complex_fixtures()
        return 0
    if args.converged:
        converged_reference()
        return 0
    if args.complex_run:
        complex_run_reference()
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
