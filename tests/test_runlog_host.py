"""The JSON-lines run log (Run.log_records / Run.write_log) built from a run's
step, half-sweep and phase records, on synthetic records (host only): one
"step" record per site step and one "half_sweep" record per half-sweep, with
the reference's right/left labels (right for the left-to-right half-sweeps)."""
import json

import numpy as np

from dmrgcc_b200 import capi


def _records():
    steps = {"half_sweep": np.array([0, 0, 1, 1], np.int32), "site": np.array([0, 1, 1, 0], np.int32),
             "energy": np.array([-1.0, -1.5, -1.6, -1.61]), "lanczos_dim": np.array([12, 30, 25, 0], np.int32),
             "discarded": np.array([1e-6, 2e-7, 0.0, 3e-9]), "psi_dim": np.array([40, 120, 120, 40], np.int64),
             "seconds": np.array([0.01, 0.02, 0.02, 0.01])}
    energies, seconds = np.array([-1.5, -1.61]), np.array([0.03, 0.03])
    phases = np.arange(10, dtype=float).reshape(2, 5) * 1e-3
    return capi.run_log_records(steps, energies, seconds, phases, np.array([3, 2], np.int32))


def test_records():
    recs = _records()
    assert [r["record"] for r in recs] == ["step"] * 4 + ["half_sweep"] * 2
    assert recs[1] == {"record": "step", "half_sweep": 0, "site": 1, "energy": -1.5, "lanczos_dim": 30,
                       "discarded": 2e-7, "psi_dim": 120, "seconds": 0.02}
    h0, h1 = recs[4], recs[5]
    assert (h0["direction"], h1["direction"]) == ("right", "left")
    assert h1["energy"] == -1.61 and h1["svd_sweeps"] == 2
    assert list(h0["phase_seconds"]) == list(capi.Run.PHASES)
    assert h1["phase_seconds"]["canonicalisation"] == 7e-3


def test_json_lines(tmp_path):
    p = tmp_path / "run.jsonl"

    class _Run:  # what Run.write_log reads, without a device
        log_records = staticmethod(_records)

    capi.Run.write_log(_Run(), str(p))
    lines = p.read_text().strip().split("\n")
    assert [json.loads(ln) for ln in lines] == _records()
