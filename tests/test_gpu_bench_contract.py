"""bench.py's output line, on a small workload: one JSON line with the keys and types that the
benchmark's consumers read (metric, value, unit, timing and configuration fields, the end-to-end
figure with its copied bytes, the kernel launch count, the roofline of the dominant kernel, the clock
record and pirate's timing loop)."""

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_line_contract():
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--steps", "4", "--warmup", "3", "--beams", "2",
           "--rank", "12", "--npri", "3", "--nfreq", "1024", "--no-cpu-baseline", "--no-plain-fp32",
           "--no-batched", "--no-spill", "--no-sifter", "--no-streams-leg"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k, t in (("metric", str), ("value", float), ("unit", str), ("n_gpus", int), ("steps", int), ("warmup", int),
                 ("ms_per_step", float), ("higher_is_better", bool), ("scaling", str), ("dtype", str), ("data", str),
                 ("config", dict), ("e2e", dict), ("gpu_launches", int), ("roofline", dict), ("clocks", dict),
                 ("time_loop", dict), ("kernel_timing", dict)):
        assert isinstance(d[k], t), k
    assert d["steps"] == 4 and d["warmup"] == 3 and d["n_gpus"] == 1 and d["higher_is_better"] is True
    assert d["value"] > 0 and d["ms_per_step"] > 0 and "vs_baseline" in d
    assert "workload" in d["config"]
    e = d["e2e"]
    assert e["value"] > 0 and e["h2d_bytes_per_step"] > 0 and e["d2h_bytes_per_step"] > 0
    r = d["roofline"]
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["peak"] > 0
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-3
    assert d["gpu_launches"] > 0
    assert {"sm_mhz", "sm_max_mhz", "reasons"} <= set(d["clocks"])
    assert d["time_loop"]["value"] > 0
