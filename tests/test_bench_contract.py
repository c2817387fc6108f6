"""The bench's output contract, on the CPU: the reference arm's JSON line (the C++ CPU restatement of
the reference's path on the c1 cuboid), its behaviour under a multi-rank launch, the defaults of a
plain `python bench.py`, and the choice of the roofline kernel.  The GPU arm itself runs in the
GPU tests' environment only."""
import argparse
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def _run(args, env_extra=None, timeout=600):
    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    env.update(env_extra or {})
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=timeout)


def test_defaults_are_one_gpu_and_a_short_run(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert a.gpus == 1 and a.impl == "b200" and a.workload == "all"
    assert a.warmup >= 3 and 1 <= a.steps <= 50
    assert a.matrix_share == 0.0 and a.bem == "auto"
    assert bench.bem_for(a, "c2") == "hmatrix" and bench.bem_for(a, "c4x64") == "dense"


def test_reference_arm_line_on_c1():
    r = _run(["--impl", "reference", "--workload", "c1", "--steps", "2", "--warmup", "1"])
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["steps"] == 2 and d["warmup"] == 1 and d["higher_is_better"] is True
    assert d["value"] > 0 and abs(d["ms_per_step"] - 1e3 / d["value"]) <= 1e-6 * d["ms_per_step"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] == "port" and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    # the GPU arm's line carries the same config dict for the same workload
    w = bench.make_workload("c1", 0)
    bem = bench.bem_for(argparse.Namespace(bem="auto"), "c1")
    assert d["config"] == json.loads(json.dumps(bench.config_for(w, bem, 1e-7, 1, False)))


def test_reference_arm_other_ranks_exit_quietly():
    r = _run(["--impl", "reference", "--workload", "c1", "--steps", "2", "--warmup", "1"],
             {"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_roofline_kernel_is_the_largest_single_kernel():
    prof = {
        "solve_neumann": {"launches": 2, "total_ms": 9.0, "bytes_per_launch": 1e9},      # container
        "bem_matvec": {"launches": 2, "total_ms": 5.0, "bytes_per_launch": 1e9},         # group of kernels
        "cg_update_smooth": {"launches": 40, "total_ms": 0.8, "bytes_per_launch": 37.6e6},
        "cg_spmv": {"launches": 40, "total_ms": 0.5, "bytes_per_launch": 26.8e6},
        "local_llg": {"launches": 2, "total_ms": 0.0, "bytes_per_launch": 40e6},
    }
    dom, d, avg_ms, achieved = bench.roofline_of(prof)
    assert dom == "cg_update_smooth"
    assert avg_ms == pytest.approx(0.02)
    assert achieved == pytest.approx(37.6e6 / 0.02e-3 / 1e9)
