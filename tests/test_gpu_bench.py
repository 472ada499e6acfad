"""The benchmark's GPU arm on a small batch: one JSON line with the keys the
benchmark contract asks for (roofline with the measured traffic and the
step's speed of light, CPU baseline, end-to-end figure with the bytes it
copies, clocks, the library's own launch count), and a device value that
agrees with the per-step timings it reports."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_line_small_batch():
    cmd = [sys.executable, "bench.py", "--pairs", "256", "--max-photons", "200000", "--steps", "3", "--warmup", "3",
           "--serving-seconds", "0", "--no-plain", "--no-tune", "--cpu-seconds", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "roofline", "cpu_baseline", "e2e", "clocks", "gpu_launches"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["steps"] == 3 and d["warmup"] == 3 and d["value"] > 0
    assert d["config"]["workload"]
    # value = photons of the timed steps / their summed device time (the steps' batches differ a little)
    assert d["value"] * d["ms_per_step"] / 1e3 == pytest.approx(d["config"]["photons_per_step_per_gpu"], rel=0.3)
    rf = d["roofline"]
    assert 0 < rf["frac"] < 1.5 and rf["achieved"] > 0 and rf["peak"] > 0
    assert rf["traffic"] is None or rf["traffic"] > 0
    sol = rf["step_speed_of_light"]
    assert sol["steps_per_s"] > 0 and 0 < sol["frac_of_ceiling"] < 1.5
    e2e = d["e2e"]
    assert e2e["value"] > 0 and e2e["h2d_bytes_per_step"] == 256 * 80 and e2e["d2h_bytes_per_step"] > 0
    cb = d["cpu_baseline"]
    assert cb["value"] > 0 and cb["cores"] >= 1 and cb["kind"] == "port" and cb["same_batch_as_gpu"] is True
    assert d["gpu_launches"] >= 3 * 3  # scan, batched, finalize per timed step
    assert "sm_mhz" in d["clocks"] and "reasons" in d["clocks"]
