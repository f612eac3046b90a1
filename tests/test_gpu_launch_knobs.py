"""The two launch switches the engine reads from the environment change
scheduling only, never arithmetic: NLS_PDL=0 launches the step kernels without
programmatic dependent launch, NLS_SPLIT=0 runs the batch as one slot group
instead of two parallel graph branches. A small batch stepped in a child
process with each switch off equals the default run bitwise (every
trajectory's reductions depend only on its own tiles)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import PKG, ROOT

pytestmark = pytest.mark.gpu

CHILD = r"""
import os, sys
import numpy as np
sys.path.insert(0, os.environ["NLS_PKG"])
import nlsb200 as nl
from nlsb200 import workloads as W
cases = [W.kg_case(96, 10.0, T=0.2, nt=40, ns=4, k=9, seed=70 + i, kinks=(i % 2 == 0), precision=nl.FP32)
         for i in range(6)]
cases += [W.nlse_case(64, 8.0, T=0.02, nt=20, ns=2, k=12, seed=80 + i, precision=nl.FP32) for i in range(4)]
out = {}
kg = nl.Pool(nl.KG_GAUTSCHI, 2, 9, nl.FP32, capacity_points=6 * 128 * 96 + 4096, max_slots=6)
ns = nl.Pool(nl.NLSE_SS2, 2, 12, nl.FP32, capacity_points=4 * 64 * 64 + 4096, max_slots=4)
slots = [(kg if c[0].method == nl.KG_GAUTSCHI else ns, None) for c in cases]
slots = [(p, p.admit(*c)) for (p, _), c in zip(slots, cases)]
for p in (kg, ns):
    while not all(q.poll(s)[1] for q, s in slots if q is p):
        p.step(7)
    p.sync()
res = [p.release(s) for p, s in slots]
np.savez(os.environ["NLS_OUT"], *[r.traj for r in res])
print("OK")
"""


def _run(tmp_path, name, env_extra):
    out = tmp_path / f"{name}.npz"
    env = dict(os.environ, NLS_PKG=PKG, NLS_OUT=str(out), **env_extra)
    r = subprocess.run([sys.executable, "-c", CHILD], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0 and "OK" in r.stdout, r.stderr[-2000:]
    z = np.load(out)
    return [z[f"arr_{i}"] for i in range(len(z.files))]


@pytest.mark.parametrize("knob", ["NLS_PDL", "NLS_SPLIT"])
def test_launch_switch_is_bitwise_neutral(tmp_path, knob):
    base = _run(tmp_path, "default", {})
    off = _run(tmp_path, "off", {knob: "0"})
    assert len(base) == len(off) == 10
    for a, b in zip(base, off):
        assert np.all(np.isfinite(a)) and np.array_equal(a, b)
