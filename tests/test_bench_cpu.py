"""bench.py on CPU: `--impl reference` prints one JSON line with the contract's
keys (the metric, unit and config of the headline workload, the CPU baseline it
times, a zero-copy e2e, at least 3 warm-up steps) and reports the reference's
own device path beside it, or why it is unavailable (no GPU here); that arm
neither imports nor loads the engine and reports the engine arm's config;
`--gpus N` starts N ranks itself and refuses to run with fewer."""
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
    assert d["config"] == bench.workload_config(bench.K_HEADLINE, 1, bench.CFG["batch"])
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    dev = d["reference_device_path"]
    assert ("value" in dev and dev["value"] > 0) or "unavailable" in dev


PROBE = r"""
import json, os, sys
sys.path.insert(0, os.environ["NLS_ROOT"])
import bench
class A:
    steps, warmup, gpus = 1, 3, 1
rc = bench.run_reference(A, 1, 0, budget_s=5.0)
maps = open("/proc/self/maps").read()
print("PROBE " + json.dumps({"rc": rc, "engine_modules": sorted(m for m in sys.modules if m.startswith("nlsb200")),
                            "engine_so": "libnlsb200.so" in maps}))
"""


def test_reference_arm_never_touches_the_engine():
    out = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, NLS_ROOT=ROOT))
    assert out.returncode == 0, out.stderr[-2000:]
    res = json.loads([l for l in out.stdout.splitlines() if l.startswith("PROBE ")][-1][6:])
    assert res["rc"] == 0 and res["engine_modules"] == [] and res["engine_so"] is False


def test_gpus_flag_starts_its_ranks():
    """`--gpus 2` without a launcher starts two ranks (gloo on CPU); the
    reference arm runs on rank 0 only and reports n_gpus 2."""
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--impl", "reference",
                          "--steps", "1", "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=900,
                         env=env)
    assert out.returncode == 0, out.stderr[-3000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2 and d["config"]["global_batch"] == 128


def test_gpus_flag_refuses_fewer_ranks():
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--impl", "reference",
                          "--steps", "1"], cwd=ROOT, capture_output=True, text=True, timeout=120, env=env)
    assert out.returncode == 2 and "2 but 1 rank" in out.stderr
