"""The one-kernel step (k2_step_dyn) of the 2-D FP32 Gautschi pools against the
launch sequence it replaces: warps claim the items of the sequence (first
pass, Lanczos passes, f(T), final pass, ghost ring and step advance) in stage
order and run the same per-tile code, so every snapshot and velocity is
bitwise equal, for KG and phi^4 (with noise), for batches of mixed grid sizes
including admissions and releases between steps, and for k at the edges of
the register f(T) sizes (8, 12, 16).

Its waits are bounded: a pool told to stall one stage's waits (a count nothing
reaches) reports NLS_ERR_TIMEOUT at the next sync, the launch having ended by
itself, and the device stays usable for the next pool.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _nl():
    import nlsb200
    return nlsb200


def _cases(k, method=None):
    nl = _nl()
    from nlsb200 import workloads as W
    method = nl.KG_GAUTSCHI if method is None else method
    out = []
    for i, n in enumerate((97, 128, 64, 150, 33)):
        out.append(W.kg_case(n, 10.0, T=0.02 * 31, nt=31, ns=5, k=k, seed=600 + i, kinks=(i % 2 == 0),
                             method=method, precision=nl.FP32))
    if method == nl.SP4_GAUTSCHI:
        for sp, *_ in out:
            sp.seed = 77
    return out


def _run(cases, one_kernel, staggered=False):
    nl = _nl()
    cap = sum(((s.nx + 31) // 32 * 32) * s.ny for s, *_ in cases) + 256 * len(cases)
    k = cases[0][0].k
    pool = nl.Pool(cases[0][0].method, 2, k, nl.FP32, capacity_points=cap, max_slots=len(cases), segment=25,
                   final_segment=16)
    pool.set_step_kernel(one_kernel)
    res = {}
    pending = list(enumerate(cases))
    live = {}
    while pending or live:
        # admit up to three at a time so that admissions and releases happen between steps
        while pending and (not staggered or len(live) < 3):
            i, cs = pending.pop(0)
            live[i] = pool.admit(*cs)
        pool.step(4)
        for i, s in list(live.items()):
            if pool.poll(s)[1]:
                info = pool.release(s)
                res[i] = (info.traj.copy(), info.vel.copy())
                del live[i]
    if one_kernel:
        assert pool.kernels_per_step() == 1
    pool.close()
    return [res[i] for i in range(len(cases))]


@pytest.mark.parametrize("k", [8, 9, 12, 16])
def test_one_kernel_step_bitwise_equals_launch_sequence(k):
    cases = _cases(k)
    a = _run(cases, True)
    b = _run(cases, False)
    for (ta, va), (tb, vb) in zip(a, b):
        assert np.all(np.isfinite(ta)) and np.array_equal(ta, tb) and np.array_equal(va, vb)


def test_one_kernel_step_phi4_and_staggered_admission():
    nl = _nl()
    cases = _cases(10, nl.SP4_GAUTSCHI)
    a = _run(cases, True, staggered=True)
    b = _run(cases, False, staggered=True)
    for (ta, va), (tb, vb) in zip(a, b):
        assert np.array_equal(ta, tb) and np.array_equal(va, vb)


def test_one_kernel_step_against_oracle():
    from conftest import rel_l2
    from parity_util import run_oracle
    cases = _cases(9)
    got = _run(cases, True)
    for (sp, u0, v0, m, c), (traj, vel) in zip(cases, got):
        otraj, ovel = run_oracle(sp, u0, v0, m, c)
        assert rel_l2(traj, otraj) < 1e-5 and rel_l2(vel, ovel) < 1e-4


@pytest.mark.parametrize("stage", [1, 8, 10])
def test_bounded_wait_runs_out_and_is_reported(stage):
    """k = 9: stage 1 is the first Lanczos pass, 8 the f(T) solves, 10 the
    ghost ring; their waits are made unsatisfiable and limited to 1000 polls."""
    nl = _nl()
    from nlsb200._lib import NlsError
    cases = _cases(9)[:2]
    cap = sum(((s.nx + 31) // 32 * 32) * s.ny for s, *_ in cases) + 512
    pool = nl.Pool(nl.KG_GAUTSCHI, 2, 9, nl.FP32, capacity_points=cap, max_slots=2)
    pool.set_step_kernel(True)
    for cs in cases:
        pool.admit(*cs)
    pool.set_wait_limit(1000, stall_stage=stage)
    pool.step(1)
    with pytest.raises(NlsError) as err:
        pool.sync()
    assert err.value.code == -10 and "ran out" in str(err.value)
    pool.close()
    # the context is intact: a fresh pool steps and matches the launch sequence
    a = _run(cases, True)
    b = _run(cases, False)
    for (ta, _), (tb, _) in zip(a, b):
        assert np.array_equal(ta, tb)
