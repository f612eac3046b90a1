"""bench.py's reference arm on CPU: `--impl reference` prints one JSON line with
the contract's keys (the metric, unit and config of the headline workload, the
CPU baseline it times, a zero-copy e2e, at least 3 warm-up steps) and reports the reference's own device
path beside it, or why it is unavailable (no GPU here)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    for key in ("value", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling", "vs_baseline",
                "dtype", "data", "config"):
        assert key in d, key
    assert d["value"] > 0 and d["steps"] == 1 and d["higher_is_better"] is True
    assert d["warmup"] >= 3  # the bench raises the warm-up to at least 3 steps
    assert "workload" in d["config"] and d["config"]["grid"] == [300, 300]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    dev = d["reference_device_path"]
    assert ("value" in dev and dev["value"] > 0) or "unavailable" in dev
