"""The batched U/t scan: many independent Bose-Hubbard chains run side by side.

The workload is 64 open chains of the reference's
real spinless Bose-Hubbard model, drawn with numpy's default_rng(0): length L
uniform in {12, 16, 20, 24, 28, 32}, U/t uniform in [1, 20], n_max = 3 (d = 4),
unit filling (N = L), bond dimension up to 128, 6 sweeps.  Each instance is an
input file of the reference's format (model/input_spinless_bose_square); the
reference runs one per process (model/real_spinless_bose_square_model.cc:11-42),
the library runs all of them side by side through dmrg_run_execute_many (each
instance on its own context and stream).

The reference's Hamiltonian has U n(n-1) with no 1/2
(model/hamiltonian/real_spinless_bose_square_hamiltonian.cc:56), so the input
file carries U_ref = U/2 for an on-site term U/2 n(n-1); hopping Jx = -t = -1.

    python -m dmrgcc_b200.scan --write DIR   # the 64 input files
"""
from __future__ import annotations

import argparse
import os

import numpy as np

LENGTHS = (12, 16, 20, 24, 28, 32)
N_INSTANCES = 64
SEED = 0
# maxm, noise per half-sweep: D ramp 32 -> 64 -> 128, noise 4..8 then off (6 sweeps)
SWEEPS = [(32, 4), (32, 4), (64, 5), (64, 5), (128, 6), (128, 6), (128, 7), (128, 7), (128, 8), (128, 8),
          (128, -1), (128, -1)]


def instances(n: int = N_INSTANCES, seed: int = SEED) -> list[dict]:
    """[{"L", "U"}] of the scan, U in units of t."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        L = int(rng.choice(LENGTHS))
        U = float(rng.uniform(1.0, 20.0))
        out.append({"L": L, "U": U})
    return out


def input_text(L: int, U: float) -> str:
    rows = "\n".join(f"        {m:<5d} 100   100    1E-12   {z}" for m, z in SWEEPS)
    return f"""input
{{
    num_site_x = {L}
    num_site_y = 1
    num_boson = {L}
    physics_dim = 4
    flux = 0.0
    Jx = -1.0
    Jy = 0.0
    U = {U / 2.0:.17g}
    mu = 0.0
    period_x = false
    period_y = false

    disk_cache = false
    cache_name = .
    cache_record = false
    record_name = record.dat
    cache_resume = false
    resume_name =
    record_process = false
    process_name = process

    first_block = 100
    first_dim = 8
    num_sweep = {len(SWEEPS) // 2}
    sweeps
    {{
        maxm  maxb  niter  canpre  noise
{rows}
    }}
}}
"""


def write_inputs(directory: str, n: int = N_INSTANCES, seed: int = SEED) -> list[str]:
    os.makedirs(directory, exist_ok=True)
    paths = []
    for i, inst in enumerate(instances(n, seed)):
        p = os.path.join(directory, f"scan_{i:02d}_L{inst['L']}.in")
        with open(p, "w") as f:
            f.write(input_text(inst["L"], inst["U"]))
        paths.append(p)
    return paths


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--write", required=True, metavar="DIR")
    ap.add_argument("-n", type=int, default=N_INSTANCES)
    a = ap.parse_args()
    for p in write_inputs(a.write, a.n):
        print(p)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
