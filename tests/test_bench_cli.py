"""The benchmark's command line and its reference arm, on CPU.

Per-workload defaults (tolerance, steps, time limit) and the metric name come from
bench.parse(); the reference arm (`--impl reference`) runs the compiled reference
solver on the host and must print one JSON line with the contract's keys."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _parse(monkeypatch, *argv):
    import bench
    monkeypatch.setattr(sys, "argv", ["bench.py", *argv])
    return bench.parse()


def test_workload_defaults(monkeypatch):
    import bench
    a = _parse(monkeypatch)
    assert a.workload == "refinery_learned" and a.eps == 1e-6 and a.steps == 1 and a.gpus == 1
    assert a.warmup >= 3
    # every leg of the learned workload stops on relative KKT and the objective criterion,
    # checking every 256 iterations, and the one-LP-per-solve FP64 comparison runs 8 instances
    assert a.eps_objective == 1e-6 and a.check_every == 256 and a.single_sample == 8
    a = _parse(monkeypatch, "--workload", "block_angular")
    assert a.eps == 1e-6 and a.steps == 5 and a.time_limit == 0.0 and a.e2e_steps == 5
    a = _parse(monkeypatch, "--workload", "ill_conditioned")
    assert a.eps == 1e-8 and a.steps == 1 and a.time_limit == 1200.0
    assert bench.metric_for(a) == "LPs/sec to 1e-08 rel KKT"
    a = _parse(monkeypatch, "--workload", "ill_conditioned", "--eps", "1e-6", "--e2e-steps", "0")
    assert a.eps == 1e-6 and a.e2e_steps == 0


def test_reference_arm_json_line():
    from oracle_lib import REF_DIR
    if not (REF_DIR / "libbharatopt_ref.so").exists():
        pytest.skip("compiled reference (oracle/_ref/libbharatopt_ref.so) not present")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--workload", "random_sparse",
                        "--steps", "1", "--warmup", "0", "--cpu-sample-iters", "4"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]


def test_learned_plan_fits_driver_command(monkeypatch):
    """The fixed driver command (--steps 20 --warmup 5) on the full configuration
    (20k labels, 600 epochs, 2k held-out) plans within 1,200 s: only the value leg
    repeats --steps times, the comparison and e2e legs run their own small counts."""
    import bench
    a = _parse(monkeypatch, "--steps", "20", "--warmup", "5")
    assert a.train_count == 20000 and a.epochs == 600 and a.heldout == 2000
    assert a.compare_steps == 1 and a.e2e_steps == 1
    plan = bench.planned_wall_s(a)
    assert plan <= 1200.0, plan
    # the value leg is what grows with --steps
    b = _parse(monkeypatch, "--steps", "21", "--warmup", "5")
    assert bench.planned_wall_s(b) - plan == pytest.approx(bench.LEARNED_LEG_S["learned"])
