"""Device energy / mass diagnostics (nls_pool_set_diagnostics).

Snapshot 0 is checked against the golden outputs of the reference's own
functions (tests/golden/diagnostics.npz, scripts/compare_utils_real_2d.py:112-131,
scripts/compare_utils_complex_2d.py:134-151); later snapshots against the
oracle's restatement applied to the snapshots the engine returned.

Tolerances (relative, per entry): FP64 pool 1e-12 (summation order only);
FP32 pool 1e-6 (m and c are stored in FP32).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "diagnostics.npz")


def _nl():
    import nlsb200
    return nlsb200


def _close(got, want, rtol):
    scale = np.maximum(np.abs(want), 1e-300)
    err = np.abs(got - want) / scale
    err[np.abs(want) == 0] = np.abs(got[np.abs(want) == 0])
    assert np.all(err < rtol), (got, want, err)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_snapshot0_matches_reference_functions(prec):
    nl = _nl()
    from oracle import diagnostics as D
    g = np.load(GOLD)
    P = nl.FP64 if prec == "fp64" else nl.FP32
    rtol = 1e-12 if prec == "fp64" else 1e-6
    for i in range(2):
        nx, ny, Lx, Ly = g[f"kg{i}_geom"]
        spec = nl.Spec(nl.KG_GAUTSCHI, 2, nx=int(nx), ny=int(ny), Lx=Lx, Ly=Ly, T=0.02, nt=2, ns=2,
                       k=8, precision=P)
        u, v, m, c = g[f"kg{i}_u"], g[f"kg{i}_v"], g[f"kg{i}_m"], g[f"kg{i}_c"]
        with nl.Solver(spec, u, v, m, c) as s:
            s.enable_diagnostics()
            s.run()
            diag = s.diagnostics()
            traj, vel = s.snapshots()
        _close(diag[0], g[f"kg{i}_diag"], rtol)
        _close(diag[1], D.kg(traj[1], vel[1], m, c, (Ly, Lx)), rtol)
        nx, ny, Lx, Ly = g[f"nlse{i}_geom"]
        spec = nl.Spec(nl.NLSE_SS2, 2, nx=int(nx), ny=int(ny), Lx=Lx, Ly=Ly, T=0.002, nt=2, ns=2,
                       k=10, precision=P)
        u = g[f"nlse{i}_u"]
        with nl.Solver(spec, u, None, np.ones(u.shape)) as s:
            s.enable_diagnostics()
            s.run()
            diag = s.diagnostics()
            traj, _ = s.snapshots()
        _close(diag[0], g[f"nlse{i}_diag"], rtol)
        _close(diag[1], D.nlse(traj[1], (Ly, Lx)), rtol)


@pytest.mark.parametrize("dim", [2, 3])
def test_pool_diagnostics_every_snapshot(dim):
    nl = _nl()
    from nlsb200 import workloads as W
    from oracle import diagnostics as D
    n = 40 if dim == 2 else 14
    spec, u0, v0, m, c = W.kg_case(n, 8.0, T=0.5, nt=50, ns=5, k=10, seed=3, dim=dim, precision=nl.FP64)
    c = 1.0 + 0.2 * np.random.default_rng(1).random(u0.shape)
    nspec, nu0, _, nm, _ = W.nlse_case(n, 6.0, T=0.05, nt=50, ns=5, k=12, seed=4, dim=dim,
                                       precision=nl.FP64)
    kp = nl.Pool(nl.KG_GAUTSCHI, dim, 10, nl.FP64, capacity_points=4 * n ** dim + 4096, max_slots=2)
    sk = kp.admit(spec, u0, v0, m, c)
    dk = kp.enable_diagnostics(sk)
    npool = nl.Pool(nl.NLSE_SS2, dim, 12, nl.FP64, capacity_points=4 * n ** dim + 4096, max_slots=2)
    sn = npool.admit(nspec, nu0, None, nm)
    dn = npool.enable_diagnostics(sn)
    for pool, slot in ((kp, sk), (npool, sn)):
        while not pool.poll(slot)[1]:
            pool.step(10)
        pool.sync()
    Ls = (8.0,) * dim
    info = kp.release(sk)
    for s in range(spec.ns):
        _close(dk[s], D.kg(info.traj[s], info.vel[s], m, c, Ls), 1e-12)
    info = npool.release(sn)
    for s in range(nspec.ns):
        _close(dn[s], D.nlse(info.traj[s], (6.0,) * dim), 1e-12)
    kp.close()
    npool.close()
