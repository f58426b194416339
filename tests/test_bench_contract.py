"""The bench's JSON contract on the CPU: the reference arm (the oracle port
timed on the host cores) prints one line with the metric, the CPU baseline
description and an e2e block without copies; the roofline helper turns
event-timed launches into achieved GB/s against the measured peak."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_reference_arm_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["unit"] == "particle-steps/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    assert line["config"]["workload"] == "mcc128"


def test_roofline_helper():
    import bench
    # 4 launches of 1e8 particles in 10 ms total: 57 B x 1e8 / 2.5 ms = 2.28 TB/s
    timers = {"push_mixed": (10.0, 4), "other": (1.0, 1)}
    r = bench._roofline(timers, "push_mixed", 57.0, 4e8)
    assert abs(r["achieved"] - 57.0 * 1e8 / 2.5e-3 / 1e9) < 1e-6
    assert abs(r["frac"] - r["achieved"] / r["peak"]) < 1e-12
    assert r["bound"] == "hbm" and r["unit"] == "GB/s" and r["kernel"] == "push_mixed"
    assert abs(r["traffic"] - bench.MEASURED_TRAFFIC_PER_PARTICLE["push_mixed"] * 1e8) < 1.0
