"""Parity at the sizes of the reference configurations (the headline metric's
cases), FP32 engine against the FP64 oracle.

  cfg1: KG 2-D 128^2, L = 10, dt = 0.01, 1000 steps, 10 snapshots, k = 10 (full length)
  cfg3 shape: NLSE 2-D SS2 batch of 200^2 grids, dt = 1e-3, k = 12 (shortened run)
  cfg4 shape: KG 3-D batch (reduced grid; the oracle cannot run 220^3 here)
  cfg2 size: 64 x 300^2 through the pool; checked by properties that do not need
             the oracle at full size (every trajectory equals its run alone,
             bitwise) plus the oracle on trajectories of the batch

Tolerance: rel-L2 <= 1e-5 on every snapshot (the metric's bound is the last one).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL32 = 1e-5


def _nl():
    import nlsb200
    return nlsb200


def _oracle(spec, u0, v0, m, c):
    from parity_util import run_oracle
    return run_oracle(spec, u0, v0, m, c)


def test_cfg1_full_length_fp32():
    nl = _nl()
    from nlsb200 import workloads as W
    cfg = W.CONFIGS["kg2d_128_fp64"]
    spec, u0, v0, m, c = W.kg_case(cfg["n"], cfg["L"], cfg["T"], cfg["nt"], cfg["ns"], k=cfg["k"], seed=1,
                                   precision=nl.FP32)
    with nl.Solver(spec, u0, v0, m) as s:
        s.run()
        traj, vel = s.snapshots()
    otraj, ovel = _oracle(spec, u0, v0, m, c)
    assert np.all(np.isfinite(traj))
    errs = [rel_l2(traj[i], otraj[i]) for i in range(spec.ns)]
    assert max(errs) < TOL32, errs
    assert rel_l2(traj[-1], otraj[-1]) < TOL32


def test_cfg3_shape_nlse_batch_fp32():
    nl = _nl()
    from nlsb200 import workloads as W
    cases = [W.nlse_case(200, 10.0, T=0.2, nt=200, ns=5, k=12, seed=40 + i, precision=nl.FP32) for i in range(3)]
    pool = nl.Pool(nl.NLSE_SS2, 2, 12, nl.FP32, capacity_points=3 * 224 * 200 + 4096, max_slots=3)
    slots = [pool.admit(sp, u0, None, m) for sp, u0, _, m, _ in cases]
    while not all(pool.poll(s)[1] for s in slots):
        pool.step(20)
    pool.sync()
    for (sp, u0, _, m, c), s in zip(cases, slots):
        info = pool.release(s)
        otraj, _ = _oracle(sp, u0, None, m, c)
        assert rel_l2(info.traj, otraj) < TOL32
    pool.close()


def test_cfg4_shape_kg3d_batch_fp32():
    nl = _nl()
    from nlsb200 import workloads as W
    cases = [W.kg_case(36, 10.0, T=0.4, nt=40, ns=4, k=10, seed=50 + i, dim=3, precision=nl.FP32) for i in range(2)]
    pool = nl.Pool(nl.KG_GAUTSCHI, 3, 10, nl.FP32, capacity_points=2 * 64 * 36 * 36 + 4096, max_slots=2)
    slots = [pool.admit(*cs) for cs in cases]
    while not all(pool.poll(s)[1] for s in slots):
        pool.step(10)
    pool.sync()
    for (sp, u0, v0, m, c), s in zip(cases, slots):
        info = pool.release(s)
        otraj, ovel = _oracle(sp, u0, v0, m, c)
        assert rel_l2(info.traj, otraj) < TOL32
        assert rel_l2(info.vel, ovel) < 1e-4
    pool.close()


def test_cfg2_size_batch_properties():
    """64 x 300^2 (the bench workload), 60 steps: every trajectory checked
    against the same trajectory run alone (bitwise) for two members, and
    against the oracle for one, with the whole batch finite."""
    nl = _nl()
    from nlsb200 import workloads as W
    B, n, nt, ns = 64, 300, 61, 3
    cases = [W.kg_case(n, 15.0, T=0.005 * nt, nt=nt, ns=ns, k=9, seed=1000 + i, kinks=(i % 2 == 0),
                       precision=nl.FP32) for i in range(B)]
    cap = B * 320 * 300 + 256 * B
    pool = nl.Pool(nl.KG_GAUTSCHI, 2, 9, nl.FP32, capacity_points=cap, max_slots=B)
    slots = [pool.admit(*cs) for cs in cases]
    assert None not in slots
    while not all(pool.poll(s)[1] for s in slots):
        pool.step(20)
    pool.sync()
    infos = [pool.release(s) for s in slots]
    pool.close()
    for info in infos:
        assert np.all(np.isfinite(info.traj)) and np.all(np.isfinite(info.vel))
    for i in (5, 62):
        sp, u0, v0, m, c = cases[i]
        with nl.Solver(sp, u0, v0, m) as s:
            s.run()
            traj, vel = s.snapshots()
        assert np.array_equal(traj, infos[i].traj) and np.array_equal(vel, infos[i].vel)
    sp, u0, v0, m, c = cases[17]
    otraj, _ = _oracle(sp, u0, v0, m, c)
    assert rel_l2(infos[17].traj, otraj) < TOL32


def test_sewi_reference_order_diverges_and_is_reported():
    """The reference's SEWI operand order (sewi_variant 0, nlse_dev.hpp:225-229)
    grows without bound on these inputs (the FP64 oracle reaches |u| ~ 1e138 by
    step 8 and then fails); the engine reports the divergence as
    NLS_ERR_NUMERIC naming the corrected order, which runs cleanly."""
    nl = _nl()
    from nlsb200 import workloads as W
    from nlsb200._lib import NlsError
    spec, u0, _, m, c = W.nlse_case(64, 10.0, T=0.02, nt=20, ns=2, k=12, seed=0, precision=nl.FP32)
    spec.method = nl.NLSE_SEWI
    spec.sewi_variant = 0
    with pytest.raises(NlsError) as err:
        with nl.Solver(spec, u0, None, m) as s:
            s.run()
            s.snapshots()
    assert err.value.code == -8 and "diverged" in str(err.value) and "variant 1" in str(err.value)
    spec.sewi_variant = 1
    with nl.Solver(spec, u0, None, m) as s:
        s.run()
        traj, _ = s.snapshots()
    assert np.all(np.isfinite(traj)) and np.abs(traj).max() < 10
