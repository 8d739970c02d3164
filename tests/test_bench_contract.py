"""bench.py's reference arm (the oracle port on the host cores) prints one
JSON line with every key of the benchmark contract; runs on CPU."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--scale", "13",
                          "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "edges/s" and d["value"] > 0
    assert d["steps"] == 2 and d["warmup"] == 1 and d["higher_is_better"] is True
    assert d["config"]["workload"] == "rmat22_ef16_exact_count"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


@pytest.mark.gpu
def test_our_arm_json_line_small_scale(tchll):
    """Our arm at R-MAT scale 16: every contract key, the oracle parity check
    passed (exact count equal, else the run fails), and any roofline fraction
    it reports is physical (<= 1.2 of the measured peak)."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--scale", "16", "--steps", "3",
                          "--warmup", "3", "--no-extras", "--cpu-seconds", "1"], capture_output=True, text=True,
                         timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "e2e", "roofline", "cpu_baseline", "gpu_launches", "clocks",
              "parity"):
        assert k in d, k
    assert d["parity"]["match"] and d["parity"]["exact_match"]
    assert d["config"]["triangles"] == d["parity"]["oracle_exact"]
    assert d["e2e"]["h2d_bytes_per_step"] > 0 and d["e2e"]["d2h_bytes_per_step"] == 64
    assert d["gpu_launches"] > 0
    frac = d["roofline"].get("frac")
    assert frac is None or 0.0 < frac <= 1.2
