"""GPU parity: the sm_100a engine (through the C ABI) against the FP64 oracle
on the same seeded inputs.

Tolerances (rel-L2 over all snapshots):
  FP64 engine : 1e-9   (same algorithm, different summation order and no CGS pass)
  FP32 engine : 1e-5   (the target tolerance at the final snapshot)
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL64 = 1e-9
TOL32 = 1e-5


def _nl():
    import nlsb200
    return nlsb200


def _run_engine(spec, u0, v0, m, c):
    nl = _nl()
    with nl.Solver(spec, u0, v0, m, c) as s:
        s.run()
        return s.snapshots()


def _cases():
    from nlsb200 import workloads as W
    from nlsb200.solver import (FP32, FP64, KG_GAUTSCHI, KG_SV, NLSE_SEWI, NLSE_SS2,
                                SP4_GAUTSCHI, SP4_SV)
    return W, FP32, FP64, KG_GAUTSCHI, KG_SV, SP4_SV, SP4_GAUTSCHI, NLSE_SS2, NLSE_SEWI


def _check(spec, u0, v0, m, c, tol, vel_tol=None):
    from parity_util import run_oracle
    traj, vel = _run_engine(spec, u0, v0, m, c)
    otraj, ovel = run_oracle(spec, u0, v0, m, c)
    assert np.all(np.isfinite(traj))
    e = rel_l2(traj, otraj)
    ef = rel_l2(traj[-1], otraj[-1])
    assert e < tol and ef < tol, (e, ef)
    if vel is not None:
        ev = rel_l2(vel, ovel)
        assert ev < (vel_tol or tol), ev
    return e


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("dim", [2, 3])
def test_kg_gautschi(prec, dim):
    W, FP32, FP64, KG, *_ = _cases()
    n = 40 if dim == 2 else 14
    spec, u0, v0, m, c = W.kg_case(n, 10.0, T=1.0, nt=100, ns=5, k=10, seed=1, dim=dim,
                                   precision=FP64 if prec == "fp64" else FP32)
    _check(spec, u0, v0, m, c, TOL64 if prec == "fp64" else TOL32,
           vel_tol=1e-9 if prec == "fp64" else 1e-4)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_kg_gautschi_anisotropic_nonzero_v0(prec):
    W, FP32, FP64, KG, *_ = _cases()
    spec, u0, v0, m, c = W.kg_case(33, 8.0, T=0.6, nt=60, ns=6, k=8, seed=2,
                                   precision=FP64 if prec == "fp64" else FP32)
    rng = np.random.default_rng(3)
    c = 1 + 0.4 * rng.random(u0.shape)
    v0 = 0.3 * np.sin(np.linspace(0, 3, u0.size)).reshape(u0.shape)
    _check(spec, u0, v0, m, c, TOL64 if prec == "fp64" else TOL32,
           vel_tol=1e-9 if prec == "fp64" else 1e-4)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("dim", [2, 3])
def test_kg_sv(prec, dim):
    W, FP32, FP64, KG, KG_SV, *_ = _cases()
    n = 40 if dim == 2 else 14
    spec, u0, v0, m, c = W.kg_case(n, 10.0, T=1.0, nt=200, ns=5, k=10, seed=4, dim=dim,
                                   method=KG_SV, precision=FP64 if prec == "fp64" else FP32)
    _check(spec, u0, v0, m, c, TOL64 if prec == "fp64" else TOL32,
           vel_tol=1e-9 if prec == "fp64" else 1e-4)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("method", ["sv", "gautschi"])
def test_phi4_with_noise(prec, method):
    W, FP32, FP64, KG, KG_SV, SP4_SV, SP4_G, *_ = _cases()
    spec, u0, v0, m, c = W.kg_case(32, 10.0, T=0.5, nt=100, ns=5, k=10, seed=5,
                                   method=SP4_SV if method == "sv" else SP4_G,
                                   precision=FP64 if prec == "fp64" else FP32)
    spec.seed = 12345
    _check(spec, u0, v0, m, c, 1e-8 if prec == "fp64" else TOL32,
           vel_tol=1e-7 if prec == "fp64" else 2e-4)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("dim", [2, 3])
def test_nlse_ss2(prec, dim):
    W, FP32, FP64, *rest = _cases()
    NLSE_SS2 = rest[-2]
    n = 32 if dim == 2 else 12
    spec, u0, v0, m, c = W.nlse_case(n, 8.0, T=0.1, nt=100, ns=5, k=12, seed=6, dim=dim,
                                     precision=FP64 if prec == "fp64" else FP32)
    _check(spec, u0, None, m, c, TOL64 if prec == "fp64" else TOL32)


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_nlse_sewi(prec, variant):
    W, FP32, FP64, *rest = _cases()
    NLSE_SEWI = rest[-1]
    # the reference operand order maps u to ~ -m|u|^2 u each step (|u| -> |u|^3),
    # so it is exercised on a few steps with |u| <= 1; the corrected form runs longer
    nt, ns = (5, 5) if variant == 0 else (20, 4)
    spec, u0, v0, m, c = W.nlse_case(28, 8.0, T=1e-3 * nt, nt=nt, ns=ns, k=10, seed=7,
                                     method=NLSE_SEWI, precision=FP64 if prec == "fp64" else FP32)
    if variant == 0:
        u0 = u0 / np.abs(u0).max()
    spec.sewi_variant = variant
    _check(spec, u0, None, m, c, TOL64 if prec == "fp64" else TOL32)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("kind", ["kg", "sv", "nlse"])
def test_multi_strip_wide_grid(prec, kind):
    """Grids wider than one warp strip (120 float / 60 double or complex-float /
    28 complex-double columns) exercise the strip halos and the slot reduction
    over many tiles."""
    W, FP32, FP64, KG, KG_SV, *rest = _cases()
    p = FP64 if prec == "fp64" else FP32
    if kind == "nlse":
        spec, u0, v0, m, c = W.nlse_case(131, 10.0, T=0.02, nt=20, ns=4, k=10, seed=9, precision=p)
    else:
        spec, u0, v0, m, c = W.kg_case(131, 10.0, T=0.2, nt=20, ns=4, k=10, seed=9, precision=p,
                                       method=KG if kind == "kg" else KG_SV)
    _check(spec, u0, v0, m, c, TOL64 if prec == "fp64" else TOL32,
           vel_tol=1e-9 if prec == "fp64" else 1e-4)


def test_batch_alone_equals_mixed():
    """Each trajectory's tiling and reduction order depend only on itself:
    results are bitwise identical alone and inside a batch of uneven sizes."""
    nl = _nl()
    W, FP32, FP64, KG, *_ = _cases()
    cases = [W.kg_case(n, 10.0, T=0.5, nt=50, ns=5, k=9, seed=s) for n, s in
             [(30, 1), (47, 2), (64, 3)]]
    alone = []
    for spec, u0, v0, m, c in cases:
        alone.append(_run_engine(spec, u0, v0, m, c)[0])
    pool = nl.Pool(KG, 2, 9, FP32, capacity_points=sum(s.n for s, *_ in cases) * 2, max_slots=4)
    slots = [pool.admit(*cs) for cs in cases]
    pool.step(49)
    pool.sync()
    for s, a in zip(slots, alone):
        info = pool.release(s)
        assert np.array_equal(info.traj, a)
    pool.close()
