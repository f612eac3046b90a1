"""Throughput against the reference's own per-trajectory FP64 GPU path, on the
same GPU: the target is that the batched FP32 engine reaches at least 10x the
grid-point-steps/s of the plain per-trajectory FP64 path.

The plain path is the reference's KG Gautschi step (device/include/kg_single.cuh
step, with the matrix functions of matfunc_real.hpp) compiled from its sources
into oracle/_ref/libref_kg.so; its step loop is timed with CUDA events, after a
warm-up run, on
- the plain configuration: 128^2 on [-10,10]^2, k = 10, dt = 0.01 (100 steps);
- one trajectory of the batched configuration's grid: 300^2 on [-15,15]^2,
  dt = 0.005 (50 steps).
The engine runs the batched configuration, 64 x 300^2, FP32, k = 10 (20 timed
steps after 3 warm-up steps), and its own plain FP64 path on the 128^2 case.
The numbers are printed (pytest -s) and the 10x target is asserted against both
reference runs.
"""
import numpy as np
import pytest

from test_gpu_reference_pin import run_ref

pytestmark = pytest.mark.gpu


def _ref_rate(n, L, dt, steps):
    import nlsb200 as nl
    from nlsb200 import workloads as W
    for nt in (3, steps + 1):  # a warm-up run, then the timed run
        spec, u0, v0, m, _ = W.kg_case(n, L, T=nt * dt, nt=nt, ns=1, k=10, seed=5, precision=nl.FP64)
        _, _, ms = run_ref(spec, u0, v0, m, 0)
    return spec.n * steps / (ms / 1e3), ms / steps


def _pool_rate(cases, precision, steps, warmup):
    from nlsb200.solver import KG_GAUTSCHI, Pool
    cap = sum(((s.nx + 31) // 32 * 32) * s.ny for s, *_ in cases) + 256 * len(cases)
    pool = Pool(KG_GAUTSCHI, 2, 10, precision, capacity_points=cap, max_slots=len(cases))
    try:
        for cs in cases:
            assert pool.admit(*cs) is not None
        pool.step(warmup)
        ms = pool.step_timed(steps)
        pool.sync()
    finally:
        pool.close()
    return sum(s.n for s, *_ in cases) * steps / (ms / 1e3), ms / steps


def test_batched_fp32_vs_reference_plain_fp64():
    import nlsb200 as nl
    from nlsb200 import workloads as W
    ref128, ref128_ms = _ref_rate(128, 10.0, 0.01, 100)
    ref300, ref300_ms = _ref_rate(300, 15.0, 0.005, 50)
    plain = [W.kg_case(128, 10.0, T=10.0, nt=1000, ns=10, k=10, seed=5, precision=nl.FP64)]
    ours64, ours64_ms = _pool_rate(plain, nl.FP64, 100, 3)
    batch = [W.kg_case(300, 15.0, T=30.0, nt=6000, ns=50, k=10, seed=i, kinks=(i % 2 == 0), precision=nl.FP32)
             for i in range(64)]
    ours32, ours32_ms = _pool_rate(batch, nl.FP32, 20, 3)
    print(f"\nreference plain FP64 128^2: {ref128_ms:.3f} ms/step, {ref128:.3e} gp-steps/s")
    print(f"reference plain FP64 300^2: {ref300_ms:.3f} ms/step, {ref300:.3e} gp-steps/s")
    print(f"engine plain FP64 128^2:    {ours64_ms:.3f} ms/step, {ours64:.3e} gp-steps/s")
    print(f"engine batched FP32 64x300^2: {ours32_ms:.3f} ms/step, {ours32:.3e} gp-steps/s")
    print(f"batched FP32 / reference plain FP64: {ours32 / ref128:.0f}x (128^2), {ours32 / ref300:.0f}x (300^2)")
    assert np.isfinite(ours32) and ours32 >= 10 * ref128 and ours32 >= 10 * ref300
