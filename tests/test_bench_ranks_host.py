"""The multi-rank path of bench.py on CPU: two `gloo` ranks on 127.0.0.1.

`bench.py --gpus N` runs N replicas (one process per GPU, no collective on the
data path); its only collectives are the barriers and the max-over-ranks of the
timed totals, after which `value` is all ranks' work over the slowest rank's
time.  These tests run that reduction and the throughput formula in two
processes, and check that the reference arm does no work on ranks other than 0.
The last test covers the bench's truncation summary of a run's step records."""
import contextlib
import io
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int) -> None:
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = [120.0, 80.0][rank]  # rank 0 is the slower replica
        dist.barrier()
        total = bench.max_over_ranks(local_ms, dist, "cpu")
        assert total == 120.0, total
        e2e = bench.max_over_ranks([3.0, 5.0][rank], dist, "cpu")
        assert e2e == 5.0, e2e
        # 2 replicas x 10 steps x 3.6e9 FLOP in 120 ms
        v = bench.whole_job_tflops(world, 3.6e9, 10, total)
        assert abs(v - 2 * 10 * 3.6e9 / 0.120 * 1e-12) < 1e-12, v
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value_two_gloo_ranks():
    mp.start_processes(_rank_main, args=(2, _free_port()), nprocs=2, join=True, start_method="spawn")


def test_single_process_reduction_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(7.5) == 7.5
    assert bench.whole_job_tflops(1, 1e12, 1, 1000.0) == pytest.approx(1.0)


def test_reference_arm_does_nothing_on_other_ranks(monkeypatch):
    """Under torchrun only rank 0 times the reference's CPU path and prints its
    line; every other rank returns at once, printing nothing."""
    import argparse

    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    called = []
    monkeypatch.setattr(bench, "cpu_reference", lambda *a, **k: called.append(a) or {})
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(argparse.Namespace(steps=3, warmup=3, gpus=2))
    assert buf.getvalue() == "" and not called


def test_truncation_summary_of_a_run_record():
    """The bench's truncation figures from a run's step records (the arrays that
    dmrg_run_steps returns): the total discarded weight and that of the last
    sweep (its two half-sweeps)."""
    import numpy as np

    sys.path.insert(0, ROOT)
    import bench

    class _Run:
        def steps(self):
            return {"half_sweep": np.array([0, 0, 1, 1, 2, 2, 3, 3], np.int32),
                    "discarded": np.array([1e-3, 2e-3, 1e-4, 1e-4, 1e-6, 2e-6, 3e-7, 4e-7])}

    t = bench.truncation_summary(_Run())
    assert t["discarded_weight_total"] == pytest.approx(3.2037e-3)
    assert t["discarded_weight_last_sweep"] == pytest.approx(3.7e-6)

    class _Broken:
        def steps(self):
            raise RuntimeError("no records")

    assert bench.truncation_summary(_Broken())["discarded_weight_total"] is None


class _FakeRun:
    """Stands in for capi.Run (the calls sweep_time and two_site_form make)."""

    PHASES = ("lanczos", "expansion", "canonicalisation", "environment", "match_merge")

    def __init__(self, ctx, path, verbose=0, precision=0, two_site=False, **kw):
        import numpy as np

        self.np = np
        self.scale = 1.0 + 0.1 * precision + 0.2 * bool(two_site)

    def execute(self):
        pass

    def half_sweeps(self):
        e = self.np.array([-45.0, -45.6, -45.65, -45.653])
        return e - 1e-9 * self.scale, self.np.array([0.5, 0.6, 0.7, 0.8]) * self.scale

    def phases(self):
        return self.np.ones((4, 5)) * 0.1 * self.scale, self.np.array([3, 4, 5, 6], self.np.int32)

    def steps(self):
        return {"half_sweep": self.np.array([0, 1, 2, 3], self.np.int32),
                "discarded": self.np.array([1e-6, 1e-7, 1e-8, 1e-9]) * self.scale}

    def close(self):
        pass


def test_sweep_sections_of_the_bench_line(monkeypatch):
    """sweep_pair and two_site_form assemble their JSON objects (times, phases,
    energies, truncation summaries, split deltas) from the run records; here
    the runs are stand-ins, so only the host logic of the bench is exercised."""
    import json

    sys.path.insert(0, ROOT)
    import bench
    from dmrgcc_b200 import capi

    monkeypatch.setattr(capi, "Run", _FakeRun)
    monkeypatch.setattr(bench, "reference_sweep_sample", lambda ctx, threads: {"unavailable": "stand-in"})
    sp = bench.sweep_pair(None)
    json.dumps(sp)
    assert sp["per_sweep_s"] == pytest.approx([1.1, 1.5])
    assert sp["truncation"]["discarded_weight_total"] == pytest.approx(1.111e-6)
    assert sp["split"]["discarded_weight_delta_vs_fp64"] == pytest.approx(0.2 * 1.111e-6)
    assert sp["split"]["abs_dE_per_site_vs_fp64"] == pytest.approx(0.2e-9 / 32.0)
    ts = bench.two_site_form(None)
    json.dumps(ts)
    # the last sweep is half-sweeps 2 and 3
    assert ts["fp64"]["truncation"]["discarded_weight_last_sweep"] == pytest.approx(1.2 * 1.1e-8)
    assert ts["last_sweep_speedup_vs_fp64"] == pytest.approx(1.2 / 1.4)


def test_scan_and_complex_sections_of_the_bench_line(monkeypatch, tmp_path):
    """scan_form and complex_form assemble their objects from stand-in runs and
    contexts (the reference binaries pointed at a missing path, so neither
    runs): the host logic only."""
    import json

    sys.path.insert(0, ROOT)
    import bench
    from dmrgcc_b200 import capi

    class _Ctx:
        def __init__(self, dev=0):
            pass

        def close(self):
            pass

    class _ScanRun(_FakeRun):
        def __init__(self, ctx, path, precision=0, **kw):
            super().__init__(ctx, path, precision=precision)

        @staticmethod
        def execute_many(runs, threads=0):
            import time

            time.sleep(0.001)

    monkeypatch.setattr(capi, "Context", _Ctx)
    monkeypatch.setattr(capi, "Run", _ScanRun)
    missing = str(tmp_path / "missing")
    monkeypatch.setattr(bench, "REF_MODEL", missing)
    monkeypatch.setattr(bench, "CPLX_MODEL", missing)
    sc = bench.scan_form(2)
    json.dumps(sc)
    assert sc["instances"] == 64 and sc["sweeps_total"] == 384
    assert sc["max_abs_dE_per_site_tf32x3_vs_fp64"] > 0 and "reference_cpu" not in sc
    cx = bench.complex_form(None, 2)
    json.dumps(cx)
    assert cx["final_energy"] == pytest.approx(-45.653 - 1e-9)
    assert "reference_final_energy" in cx and "reference_cpu_sample" not in cx
