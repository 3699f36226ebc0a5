#!/usr/bin/env python
"""Benchmark of the DMRG hot path on B200: block-sparse H_eff*psi.

Workload: one H_eff*psi (the Lanczos matvec, RealTensorContraction::
MultiplyEffectHamilton) on the block structure of the 8x4 Bose-Hubbard cylinder
(periodic in y, d=5, N=16, t=1, U=8) at bond dimension 1024, site 16, dumped from
the reference's own run (tests/golden/heff_struct_cyl8x4_D1024.nac), with seeded
synthetic values.  A step = one matvec.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--precision fp64]

The line also carries `split`: the same matvec through a DMRG_PREC_TF32X3
operator (tcgen05 tensor cores), its time and its error against the FP64 result;
and `sweep`: the wall time of one whole DMRG run of the same cylinder input (8
sweeps, D up to 1024) through dmrg_run_execute (N=1 only), in FP64 and with
TF32X3 matvecs; `two_site`: the same run with two-site sweeps; `complex`: a
whole complex run (Hofstadter 6x6); `scan`: the 64-instance U/t scan side by
side.

Multi-GPU: replicas only (each rank runs its own matvec; no collective on the
data path); value = all ranks' FLOPs / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STRUCT = os.path.join(ROOT, "tests", "golden", "heff_struct_cyl8x4_D1024.nac")
CYL_INPUT = os.path.join(ROOT, "dmrgcc_b200", "inputs", "cylinder8x4_spinless.in")
METRIC = "sweep time & H·ψ TFLOP/s, split-prec vs FP64 on 1 B200 at |ΔE/site|≤1e-10"
WORKLOAD = "H_eff*psi, 8x4 Bose-Hubbard cylinder (d=5, N=16, U=8), D=1024, site 16"
PROBE = os.path.join(ROOT, "oracle", "_ref", "probe_heff")
SEED = 2024
FLUSH_BYTES = 256 << 20  # > 126 MB L2


def bench_config(psi_dim: int, gflop: float) -> dict:
    """The workload description, identical on both arms."""
    return {"workload": WORKLOAD, "psi_dim": int(psi_dim), "gflop_per_step": round(float(gflop), 6),
            "structure": os.path.basename(STRUCT), "seed": SEED}


def profiled_traffic() -> dict | None:
    """DRAM bytes per matvec of the FP64 path (stage A + stage B launches), from
    the committed ncu summary of the same workload (a line
    `traffic_bytes_per_matvec: <bytes>` in profiles/gemm_f64_heff_cyl8x4_D1024.md)."""
    p = os.path.join(ROOT, "profiles", "gemm_f64_heff_cyl8x4_D1024.md")
    try:
        with open(p) as f:
            for line in f:
                if line.startswith("traffic_bytes_per_matvec:"):
                    return {"bytes": float(line.split(":", 1)[1]), "source": os.path.relpath(p, ROOT)}
    except OSError:
        pass
    return None


def max_over_ranks(x: float, dist=None, device: str = "cuda") -> float:
    """The maximum of `x` over every rank of the default process group (`dist`
    is torch.distributed, or None for a single process, which returns `x`).
    Every rank must call it at the same point: it is one all-reduce."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_tflops(world: int, flop_per_step: float, steps: int, max_ms: float) -> float:
    """Whole-job throughput of `world` replicas that each ran `steps` steps of
    `flop_per_step`, timed as the slowest rank's `max_ms`."""
    return world * flop_per_step * steps / (max_ms * 1e-3) * 1e-12


def peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while active."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu, self.rows, self.proc = gpu, [], None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 4 + i and r[4 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def cpu_reference(steps: int, warmup: int, threads: int) -> dict:
    """The reference's own MultiplyEffectHamilton (oracle/_ref/probe_heff, OpenBLAS)."""
    if not os.path.exists(PROBE):
        return {"unavailable": f"{PROBE} not built (make -C oracle)"}
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS=str(threads),
               PROBE_WARMUP=str(warmup))
    r = subprocess.run([PROBE, STRUCT, str(steps), str(SEED)], capture_output=True, text=True, env=env,
                       timeout=1800)
    if r.returncode != 0:
        return {"unavailable": f"probe_heff failed: {r.stderr.strip()[-200:]}"}
    return json.loads(r.stdout.strip().splitlines()[-1])


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    res = cpu_reference(args.steps, args.warmup, threads)
    if "unavailable" in res:
        print(json.dumps({"impl": "reference", "unavailable": res["unavailable"]}))
        return
    tflops = res["gflop"] / res["mean_s"] * 1e-3
    line = {
        "impl": "reference", "metric": METRIC, "value": tflops, "unit": "TFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["mean_s"] * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded splitmix64 values on the "
        "reference's own D=1024 block structure)",
        "config": bench_config(res["psi_dim"], res["gflop"]),
        "backend": "reference MultiplyEffectHamilton + OpenBLAS 0.3.15 dgemm",
        "cpu_baseline": {"value": tflops, "unit": "TFLOP/s", "cores": res["threads"], "kind": "reference",
                         "sample": f"{args.steps} H_eff*psi calls after {args.warmup} warm-up calls"},
        "e2e": {"value": tflops, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def split_form(ctx, step, psi, L, R, out_ref, steps: int, flush, stream, prec: int, name: str) -> dict:
    """The same matvec through a split-precision operator (tcgen05 tensor cores,
    TF32 or BF16 hi/lo parts): per-step time with the same L2 flush, and its
    error against the FP64 result on the same vectors."""
    import numpy as np
    import torch

    from dmrgcc_b200 import capi

    h3 = capi.Heff(ctx, step.site, step.L, step.R, precision=prec)
    h3.set_env(L, R)
    out = capi.DeviceArray(ctx, step.psi_dim)
    for _ in range(3):
        h3.apply(psi, out, accumulate=False)
    ctx.sync()
    got = out.download()
    ref = out_ref.download()
    rel = float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    for e0, e1 in evs:
        flush.zero()
        e0.record(stream)
        h3.apply(psi, out, accumulate=False)
        e1.record(stream)
    torch.cuda.synchronize()
    ctx.sync()  # reports a tensor-core wait that gave up
    ms = sum(e0.elapsed_time(e1) for e0, e1 in evs) / steps
    alg, _ = h3.flops()
    prof = [h3.profile(psi, out) for _ in range(3)]
    return {"precision": name, "value": alg / (ms * 1e-3) * 1e-12, "unit": "TFLOP/s", "ms_per_step": ms,
            "speedup_vs_fp64": None, "max_rel_err_vs_fp64": rel,
            "stage_ms": {"stage_a_with_psi_packing": float(np.mean([p[0] for p in prof])),
                         "stage_b": float(np.mean([p[1] for p in prof]))},
            "kernel": "gemm_split_kernel (tcgen05.mma kind::%s, 3 products, FP32 accumulation in TMEM)"
                      % ("f16 on bf16" if name == "bf16x3" else "tf32")}


def truncation_summary(run) -> dict:
    """The discarded weight (sum of dropped sigma^2) summed over a run's
    truncations, and over those of its last sweep, from dmrg_run_steps."""
    try:
        st = run.steps()
        hs = st["half_sweep"]
        last = hs >= (hs.max() - 1) if len(hs) else hs
        return {"discarded_weight_total": float(st["discarded"].sum()),
                "discarded_weight_last_sweep": float(st["discarded"][last].sum())}
    except Exception as e:  # a summary must not cost the bench line
        return {"discarded_weight_total": None, "error": str(e)[:200]}


def sweep_time(ctx, precision: int = 0, name: str = "fp64") -> dict:
    """One whole run of the 8x4 cylinder input (D ramp 128 -> 1024, 8 sweeps =
    16 half-sweeps, niter 100, noise on for the first 12 half-sweeps), wall
    clock on the host around dmrg_run_execute (device work + host bookkeeping),
    with the H_eff*psi products in `precision` (FP64 Lanczos, eigensolve and SVD
    in every case)."""
    from dmrgcc_b200 import capi

    run = capi.Run(ctx, CYL_INPUT, verbose=0, precision=precision)
    t0 = time.perf_counter()
    run.execute()
    total = time.perf_counter() - t0
    e, s = run.half_sweeps()
    ph, sw = run.phases()
    out = {
        "workload": "whole DMRG run, 8x4 Bose-Hubbard cylinder (d=5, N=16, U=8), D 128->1024, 8 sweeps",
        "precision": name, "total_s": total,
        "per_sweep_s": [float(s[2 * i] + s[2 * i + 1]) for i in range(len(s) // 2)],
        "phase_s": {k: float(v) for k, v in zip(capi.Run.PHASES, ph.sum(axis=0))},
        "svd_sweeps": int(sw.sum()), "final_energy": float(e[-1]),
        "truncation": truncation_summary(run),
    }
    run.close()
    return out


REF_MODEL = os.path.join(ROOT, "oracle", "_ref", "real_spinless_bose_square_model")


def first_sweep_input(path: str, out_path: str) -> None:
    """The input file with its sweep table cut to the first full sweep (two
    half-sweep rows)."""
    import re

    with open(path) as f:
        text = f.read()
    text = re.sub(r"num_sweep\s*=\s*\d+", "num_sweep = 1", text)
    head, rest = text.split("sweeps", 1)
    lines = rest.splitlines()
    out, rows = [], 0
    for ln in lines:
        tok = ln.split()
        if tok and tok[0].lstrip("-").isdigit():
            rows += 1
            if rows > 2:
                continue
        out.append(ln)
    with open(out_path, "w") as f:
        f.write(head + "sweeps" + "\n".join(out))


def reference_sweep_sample(ctx, threads: int) -> dict:
    """A bounded sample of the whole-run comparison, timed on this host: the
    first sweep (D=128) of the 8x4 cylinder input, with its initialisation, run
    by the reference (oracle/_ref, OpenBLAS, `threads` host threads) and by the
    library (dmrg_run_execute), same input file; wall times and final energies."""
    import tempfile

    from dmrgcc_b200 import capi

    if not os.path.exists(REF_MODEL):
        return {"unavailable": f"{REF_MODEL} not built (make -C oracle)"}
    with tempfile.TemporaryDirectory() as tmp:
        inp = os.path.join(tmp, "cyl8x4_first_sweep.in")
        first_sweep_input(CYL_INPUT, inp)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS=str(threads))
        t0 = time.perf_counter()
        r = subprocess.run([REF_MODEL, inp], capture_output=True, text=True, env=env, cwd=tmp, timeout=900)
        ref_wall = time.perf_counter() - t0
        if r.returncode != 0:
            return {"unavailable": f"reference run failed: {r.stderr.strip()[-200:]}"}
        ref_e = [float(ln.split("=")[1]) for ln in r.stdout.splitlines() if "energy =" in ln]
        run = capi.Run(ctx, inp, verbose=0)
        t0 = time.perf_counter()
        run.execute()
        lib_wall = time.perf_counter() - t0
        e, _ = run.half_sweeps()
        run.close()
    return {"sample": "initialisation + first sweep (D=128) of the 8x4 cylinder input, same input file",
            "cores": threads, "reference_s": ref_wall, "library_s": lib_wall, "speedup": ref_wall / lib_wall,
            "reference_energy": ref_e[-1] if ref_e else None, "library_energy": float(e[-1])}


def scan_form(threads: int) -> dict:
    """The batched U/t scan (64 seeded open chains, L in
    {12..32}, U/t in [1, 20], d=4, unit filling, D<=128, 6 sweeps): all 64 runs
    side by side on this GPU (dmrg_run_execute_many, one context and stream per
    instance), in FP64 and with TF32X3 matvecs; aggregate sweeps per second,
    per-instance |dE/site| of the TF32X3 run against the FP64 run; and the
    reference binary on the same 64 input files, one process per instance with
    one BLAS thread, `threads` at a time (the reference runs one instance per
    process)."""
    import tempfile
    from concurrent.futures import ThreadPoolExecutor

    from dmrgcc_b200 import capi, scan

    out = {"workload": "64 Bose-Hubbard chains side by side (seeded U/t scan, D<=128, 6 sweeps)"}
    with tempfile.TemporaryDirectory() as tmp:
        paths = scan.write_inputs(tmp)
        insts = scan.instances()
        res = {}
        for name, prec in (("fp64", capi.DMRG_PREC_FP64), ("tf32x3", capi.DMRG_PREC_TF32X3)):
            ctxs = [capi.Context(0) for _ in paths]
            runs = [capi.Run(c, p, precision=prec) for c, p in zip(ctxs, paths)]
            t0 = time.perf_counter()
            capi.Run.execute_many(runs, 0)
            wall = time.perf_counter() - t0
            res[name] = {"wall_s": wall, "sweeps_per_s": 6 * len(runs) / wall,
                         "energy": [float(r.half_sweeps()[0][-1]) for r in runs]}
            for r in runs:
                r.close()
            for c in ctxs:
                c.close()
        de = [abs(a - b) / i["L"] for a, b, i in zip(res["tf32x3"]["energy"], res["fp64"]["energy"], insts)]
        out.update({"instances": len(paths), "sweeps_total": 6 * len(paths),
                    "fp64": {k: v for k, v in res["fp64"].items() if k != "energy"},
                    "tf32x3": {k: v for k, v in res["tf32x3"].items() if k != "energy"},
                    "max_abs_dE_per_site_tf32x3_vs_fp64": max(de)})
        if os.path.exists(REF_MODEL):
            env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1")

            def one(p):
                r = subprocess.run([REF_MODEL, p], capture_output=True, text=True, env=env, cwd=tmp, timeout=900)
                es = [float(ln.split("=")[1]) for ln in r.stdout.splitlines() if "energy =" in ln]
                return es[-1] if es else float("nan")

            t0 = time.perf_counter()
            with ThreadPoolExecutor(max_workers=threads) as ex:
                ref_e = list(ex.map(one, paths))
            wall = time.perf_counter() - t0
            dref = [abs(a - b) / i["L"] for a, b, i in zip(res["fp64"]["energy"], ref_e, insts)]
            out["reference_cpu"] = {"wall_s": wall, "sweeps_per_s": 6 * len(paths) / wall, "cores": threads,
                                    "processes": "one per instance, 1 BLAS thread each",
                                    "max_abs_dE_per_site_fp64_vs_reference": max(dref)}
            out["speedup_vs_reference"] = out["fp64"]["sweeps_per_s"] / out["reference_cpu"]["sweeps_per_s"]
    return out


def sweep_pair(ctx) -> dict:
    """The whole run in FP64 and with TF32X3 matvecs, back to back: times, the
    split run's speedup per sweep and its final-energy difference per site
    (32 sites) against the FP64 run; plus a bounded sample of the same input
    run by the reference on this host."""
    fp64 = sweep_time(ctx)
    split = sweep_time(ctx, 2, "tf32x3")
    fp64["reference_cpu_sample"] = reference_sweep_sample(ctx, os.cpu_count() or 1)
    fp64["split"] = {"precision": "tf32x3", "total_s": split["total_s"], "per_sweep_s": split["per_sweep_s"],
                     "phase_s": split["phase_s"], "final_energy": split["final_energy"],
                     "speedup_vs_fp64": fp64["total_s"] / split["total_s"],
                     "abs_dE_per_site_vs_fp64": abs(split["final_energy"] - fp64["final_energy"]) / 32.0,
                     "truncation": split["truncation"]}
    a, b = fp64["truncation"].get("discarded_weight_total"), split["truncation"].get("discarded_weight_total")
    fp64["split"]["discarded_weight_delta_vs_fp64"] = (b - a) if a is not None and b is not None else None
    return fp64


def two_site_form(ctx) -> dict:
    """Two-site sweeps (dmrg_run_options_t.two_site) over the same cylinder input
    and sweep table, in FP64 and with TF32X3 matvecs: whole-run and per-sweep wall
    times (the last sweeps run at D=1024), phases, final energies and the split
    run's |dE/site| against the FP64 run (32 sites)."""
    from dmrgcc_b200 import capi

    res = {}
    for name, prec in (("fp64", capi.DMRG_PREC_FP64), ("tf32x3", capi.DMRG_PREC_TF32X3)):
        run = capi.Run(ctx, CYL_INPUT, verbose=0, precision=prec, two_site=True)
        t0 = time.perf_counter()
        run.execute()
        total = time.perf_counter() - t0
        e, s = run.half_sweeps()
        ph, sw = run.phases()
        res[name] = {"total_s": total, "per_sweep_s": [float(s[2 * i] + s[2 * i + 1]) for i in range(len(s) // 2)],
                     "phase_s": {k: float(v) for k, v in zip(capi.Run.PHASES, ph.sum(axis=0))},
                     "svd_sweeps": int(sw.sum()), "final_energy": float(e[-1]),
                     "truncation": truncation_summary(run)}
        run.close()
    out = {"workload": "two-site DMRG, 8x4 Bose-Hubbard cylinder (d=5, N=16, U=8), D 128->1024, 8 sweeps"}
    out.update(res)
    out["speedup_vs_fp64"] = res["fp64"]["total_s"] / res["tf32x3"]["total_s"]
    out["last_sweep_speedup_vs_fp64"] = res["fp64"]["per_sweep_s"][-1] / res["tf32x3"]["per_sweep_s"][-1]
    out["abs_dE_per_site_tf32x3_vs_fp64"] = abs(res["tf32x3"]["final_energy"] - res["fp64"]["final_energy"]) / 32.0
    return out


CPLX_INPUT = os.path.join(ROOT, "dmrgcc_b200", "inputs", "hofstadter6x6.in")
CPLX_MODEL = os.path.join(ROOT, "oracle", "_ref", "complex_spinful_bose_square_model")
CPLX_REFERENCE = os.path.join(ROOT, "tests", "golden", "hofstadter6x6_reference.txt")


def complex_form(ctx, threads: int) -> dict:
    """The complex path on the 6x6 Hofstadter geometry (periodic in y, flux
    1/6, U=10, d=3; 4 bosons, D ramp 32 -> 256, 5 sweeps;
    hofstadter6x6.in): the whole complex run (dmrg_run_execute, every tensor
    complex), its final energy against the reference's on the same input
    (tests/golden/hofstadter6x6_reference.txt, 1 BLAS thread), and the
    reference's initialisation + first sweep timed on this host beside the
    library's (`threads` BLAS threads)."""
    import tempfile

    from dmrgcc_b200 import capi

    run = capi.Run(ctx, CPLX_INPUT, verbose=0, model="complex_spinful_bose_square")
    t0 = time.perf_counter()
    run.execute()
    total = time.perf_counter() - t0
    e, s = run.half_sweeps()
    ph, _ = run.phases()
    run.close()
    out = {"workload": "complex Hofstadter 6x6 (flux 1/6, 4 bosons, d=3), D 32->256, 5 sweeps",
           "total_s": total, "phase_s": {k: float(v) for k, v in zip(capi.Run.PHASES, ph.sum(axis=0))},
           "final_energy": float(e[-1])}
    if os.path.exists(CPLX_REFERENCE):
        with open(CPLX_REFERENCE) as f:
            e_ref = float([ln.split()[1] for ln in f if ln.startswith("hofstadter6x6")][0])
        out["reference_final_energy"] = e_ref
        out["abs_dE_per_site_vs_reference"] = abs(float(e[-1]) - e_ref) / 36.0
    if os.path.exists(CPLX_MODEL):
        with tempfile.TemporaryDirectory() as tmp:
            inp = os.path.join(tmp, "h66_first_sweep.in")
            first_sweep_input(CPLX_INPUT, inp)
            env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS=str(threads))
            t0 = time.perf_counter()
            r = subprocess.run([CPLX_MODEL, inp], capture_output=True, text=True, env=env, cwd=tmp, timeout=900)
            ref_wall = time.perf_counter() - t0
            lib = capi.Run(ctx, inp, verbose=0, model="complex_spinful_bose_square")
            t0 = time.perf_counter()
            lib.execute()
            lib_wall = time.perf_counter() - t0
            lib.close()
        if r.returncode == 0:
            out["reference_cpu_sample"] = {"sample": "initialisation + first sweep (D=32) of the same input",
                                           "cores": threads, "reference_s": ref_wall, "library_s": lib_wall,
                                           "speedup": ref_wall / lib_wall}
    return out


def run_b200(args) -> None:
    import numpy as np
    import torch

    from dmrgcc_b200 import capi
    from dmrgcc_b200.problem import SiteStep

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    ctx = capi.Context(local)
    # A dedicated (non-default) stream shared by torch's events and the library's
    # launches: the events then bracket exactly the kernels they time.
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    assert ctx.stream == stream.cuda_stream != 0

    step = SiteStep.from_nac(STRUCT)
    prec = {"fp64": capi.DMRG_PREC_FP64, "tf32x3": capi.DMRG_PREC_TF32X3,
            "bf16x3": capi.DMRG_PREC_BF16X3}[args.precision]
    heff = capi.Heff(ctx, step.site, step.L, step.R, precision=prec)
    psi, L, R = step.synthetic_device(ctx, seed=SEED + rank)
    heff.set_env(L, R)
    out = capi.DeviceArray(ctx, step.psi_dim)
    out.zero()
    flush = capi.DeviceArray(ctx, FLUSH_BYTES // 8)
    alg_flops, exec_flops = heff.flops()

    fp64_dmma = ctx.fp64_peak(0)
    fp64_dfma = ctx.fp64_peak(1)
    fp64_peak = max(fp64_dmma, fp64_dfma)

    for _ in range(args.warmup):
        heff.apply(psi, out, accumulate=True)
    torch.cuda.synchronize()

    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = capi.launch_count()
    with ClockSampler(local) as clk:
        for e0, e1 in evs:
            flush.zero()  # evict L2 between timed steps (outside the event pair)
            e0.record(stream)
            heff.apply(psi, out, accumulate=True)
            e1.record(stream)
        torch.cuda.synchronize()
    launches = capi.launch_count() - launches0  # this library's kernels in the timed loop
    if dist:
        dist.barrier()
    step_ms = [e0.elapsed_time(e1) for e0, e1 in evs]
    total_ms = max_over_ranks(sum(step_ms), dist)
    ms_per_step = total_ms / args.steps
    value = whole_job_tflops(world, alg_flops, args.steps, total_ms)

    # per-launch durations (stage A: K*R products, stage B: L*(KR) sums), L2 flushed
    prof = []
    for _ in range(max(3, min(args.steps, 10))):
        flush.zero()
        prof.append(heff.profile(psi, out))
    ms_a = statistics.mean(p[0] for p in prof)
    ms_b = statistics.mean(p[1] for p in prof)

    # end to end through the host-buffer entry point (pinned host memory)
    h_psi = torch.empty(step.psi_dim, dtype=torch.float64).pin_memory()
    h_out = torch.zeros(step.psi_dim, dtype=torch.float64).pin_memory()
    h_psi.copy_(torch.from_numpy(np.linspace(-1, 1, step.psi_dim)))
    lib = capi.lib()
    for _ in range(args.warmup):
        capi.check(lib.dmrg_heff_apply_host(heff.h, h_psi.data_ptr(), h_out.data_ptr(), 0), "apply_host")
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        capi.check(lib.dmrg_heff_apply_host(heff.h, h_psi.data_ptr(), h_out.data_ptr(), 0), "apply_host")
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), dist)
    e2e_value = whole_job_tflops(world, alg_flops, args.steps, e2e_ms)

    if rank == 0:
        traffic = profiled_traffic()
        dominant = "stage_b" if ms_b >= ms_a else "stage_a"
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else args.precision + " (f32 accumulate per term, f64 sums)",
            "data": "synthetic (seeded splitmix64 values on the reference's own D=1024 block structure)",
            "config": bench_config(step.psi_dim, alg_flops * 1e-9),
            # exec_flops counts the products the schedule runs (each K*R product
            # once), not the padding of the 64x64x16 DMMA tiles around them
            "detail": {"precision": args.precision, "gflop_per_step_scheduled": exec_flops * 1e-9,
                       "gflop_note": "scheduled products without the tile padding of the DMMA tiles",
                       "l2": "256 MiB write between timed steps (outside the per-step CUDA-event pair)",
                       "parallelism": f"replicas x{world}"},
            # counted by the library (dmrg_launch_count) around the timed loop: per
            # matvec the stage A and stage B grouped GEMMs and the stage B split-K reduce
            "gpu_launches": launches,
            "e2e": {"value": e2e_value, "unit": "TFLOP/s", "h2d_bytes_per_step": step.psi_dim * 8,
                    "d2h_bytes_per_step": step.psi_dim * 8,
                    "note": "dmrg_heff_apply_host: pinned psi in, matvec, result out, sync; environments resident"},
            "roofline": {
                "bound": "tensor", "kernel": "gemm_f64_kernel (whole matvec: stage A + stage B)",
                "achieved": alg_flops / (ms_per_step * 1e-3) * 1e-12, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": alg_flops / (ms_per_step * 1e-3) * 1e-12 / fp64_peak,
                "traffic": traffic["bytes"] if traffic else None,
                "traffic_source": traffic["source"] if traffic else None,
                "peak_source": f"measured in this run: DMMA loop {fp64_dmma:.2f}, DFMA loop {fp64_dfma:.2f} TFLOP/s",
                "stage_ms": {"stage_a": ms_a, "stage_b": ms_b, "dominant": dominant},
            },
            "clocks": clk.summary(),
        }
        if args.precision == "fp64" and not args.no_split:
            ref_out = capi.DeviceArray(ctx, step.psi_dim)
            heff.apply(psi, ref_out, accumulate=False)
            line["split"] = [split_form(ctx, step, psi, L, R, ref_out, min(args.steps, 500), flush, stream, p, n)
                             for p, n in ((capi.DMRG_PREC_TF32X3, "tf32x3"), (capi.DMRG_PREC_BF16X3, "bf16x3"))]
            for sp in line["split"]:
                sp["speedup_vs_fp64"] = ms_per_step / sp["ms_per_step"]
        if world == 1 and not args.no_sweep:
            line["sweep"] = sweep_pair(ctx)
        if world == 1 and not args.no_sweep:
            line["two_site"] = two_site_form(ctx)
            line["complex"] = complex_form(ctx, os.cpu_count() or 1)
        if world == 1 and not args.no_scan:
            line["scan"] = scan_form(min(os.cpu_count() or 1, 64))
        cpu = cpu_reference(args.cpu_reps, 1, os.cpu_count() or 1) if not args.no_cpu else {"unavailable": "skipped"}
        if "unavailable" not in cpu:
            line["cpu_baseline"] = {"value": cpu["gflop"] / cpu["mean_s"] * 1e-3, "unit": "TFLOP/s",
                                    "cores": cpu["threads"], "kind": "reference",
                                    "sample": f"{cpu['reps']} H_eff*psi calls of the same workload through the "
                                              "reference's MultiplyEffectHamilton (OpenBLAS)"}
        else:
            line["cpu_baseline"] = {"value": None, "unit": "TFLOP/s", "cores": 0, "kind": "reference",
                                    "sample": cpu["unavailable"]}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--precision", choices=["fp64", "tf32x3", "bf16x3"], default="fp64")
    ap.add_argument("--cpu-reps", type=int, default=30)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-sweep", action="store_true", help="skip the whole-run sweep-time measurement")
    ap.add_argument("--no-scan", action="store_true", help="skip the 64-instance U/t scan")
    ap.add_argument("--no-split", action="store_true", help="skip the TF32X3 form of the matvec")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)
    return 0


if __name__ == "__main__":
    sys.exit(main())
