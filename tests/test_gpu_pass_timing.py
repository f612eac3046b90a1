"""Pass timing entry points (nls_pool_time_pass, nls_pool_time_passes): they
return positive durations and the grid points of one launch, reject pass
indices outside 1..k-2, and leave the state unchanged (the passes are
idempotent), so a run that was timed midway equals one that was not, bitwise."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases(nl, W, k):
    return [W.kg_case(n, 10.0, T=0.3, nt=16, ns=4, k=k, seed=300 + i, kinks=(i % 2 == 0), precision=nl.FP32)
            for i, n in enumerate((64, 97, 128, 150))]


def _run(timed):
    import nlsb200 as nl
    from nlsb200 import workloads as W
    k = 9
    cases = _cases(nl, W, k)
    cap = sum(((s.nx + 31) // 32 * 32) * s.ny for s, *_ in cases) + 256 * len(cases)
    pool = nl.Pool(nl.KG_GAUTSCHI, 2, k, nl.FP32, capacity_points=cap, max_slots=len(cases))
    slots = [pool.admit(*c) for c in cases]
    pool.step(5)
    out = {}
    if timed:
        out["iso"] = pool.time_pass(2, 3)
        out["chain"] = pool.time_passes(2, k - 2, 2)
        out["chain_lo"] = pool.time_passes(1, k - 2, 1)
        out["rep"] = pool.time_passes(3, 3, 4)
        for j0, j1 in ((0, 2), (3, 2), (2, k - 1)):
            with pytest.raises(RuntimeError):
                pool.time_passes(j0, j1, 1)
    while not all(pool.poll(s)[1] for s in slots):
        pool.step(4)
    pool.sync()
    trajs = [pool.release(s).traj.copy() for s in slots]
    pool.close()
    return trajs, out, sum(s.n for s, *_ in cases)


def test_pass_timing_leaves_the_state_unchanged():
    base, _, _ = _run(False)
    trajs, out, npts = _run(True)
    for key, (ms, pts) in out.items():
        assert ms > 0.0, key
        assert pts == npts, (key, pts, npts)
    for a, b in zip(base, trajs):
        assert np.array_equal(a, b)
