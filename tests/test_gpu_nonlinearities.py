"""The nonlinearities the reference's build names without sources
(device/CMakeLists.txt:7-29: sine-Gordon, double and hyperbolic sine-Gordon,
cubic-quintic and saturable NLSE) with the potentials of its sampler
(scripts/real_sampler.py:32-46), on the existing integrators: the engine
against the FP64 oracle on the same seeded inputs, through every kernel family
that evaluates g(u) or rho (2-D packed and generic passes, Stormer-Verlet,
3-D warp and plane kernels, FP32 and FP64, SS2 and SEWI).

Tolerance: rel-L2 over all snapshots 1e-5 (FP32) / 1e-9 (FP64); velocity 1e-4 / 1e-9.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _check(spec, u0, v0, m, c, tol, vel_tol):
    import nlsb200 as nl
    from parity_util import run_oracle
    with nl.Solver(spec, u0, v0, m, c) as s:
        s.run()
        traj, vel = s.snapshots()
    otraj, ovel = run_oracle(spec, u0, v0, m, c)
    assert np.all(np.isfinite(traj))
    e = rel_l2(traj, otraj)
    assert e < tol, e
    if vel is not None and vel_tol:
        assert rel_l2(vel, ovel) < vel_tol
    return e


KG_CASES = [  # (kind, method, dim, precision)
    ("NL_SINE", "KG_GAUTSCHI", 2, "FP32"),
    ("NL_DSINE", "KG_GAUTSCHI", 2, "FP32"),
    ("NL_SINH", "KG_GAUTSCHI", 2, "FP32"),
    ("NL_SINE", "KG_GAUTSCHI", 2, "FP64"),
    ("NL_SINE", "KG_SV", 2, "FP32"),
    ("NL_DSINE", "SP4_SV", 2, "FP32"),
    ("NL_SINH", "KG_GAUTSCHI", 3, "FP32"),
    ("NL_SINE", "KG_GAUTSCHI", 3, "FP64"),
]


@pytest.mark.parametrize("kind,method,dim,prec", KG_CASES)
def test_kg_family_kinds(kind, method, dim, prec):
    import nlsb200 as nl
    from nlsb200 import workloads as W
    n = 40 if dim == 2 else 14
    p = getattr(nl, prec)
    spec, u0, v0, m, c = W.kg_case(n, 10.0, T=0.5, nt=50, ns=5, k=10, seed=7, dim=dim, precision=p,
                                   method=getattr(nl, method))
    spec.nonlinearity = getattr(nl, kind)
    _check(spec, u0, v0, m, c, 1e-5 if p == nl.FP32 else 1e-9, 1e-4 if p == nl.FP32 else 1e-9)


NLSE_CASES = [  # (kind, method, dim, precision)
    ("NL_CQ", "NLSE_SS2", 2, "FP32"),
    ("NL_SAT", "NLSE_SS2", 2, "FP32"),
    ("NL_CQ", "NLSE_SS2", 2, "FP64"),
    ("NL_SAT", "NLSE_SEWI", 2, "FP32"),
    ("NL_CQ", "NLSE_SS2", 3, "FP32"),
]


@pytest.mark.parametrize("kind,method,dim,prec", NLSE_CASES)
def test_nlse_kinds(kind, method, dim, prec):
    import nlsb200 as nl
    from nlsb200 import workloads as W
    n = 40 if dim == 2 else 14
    p = getattr(nl, prec)
    spec, u0, _, m, c = W.nlse_case(n, 8.0, T=0.05, nt=50, ns=5, k=12, seed=8, dim=dim, precision=p)
    spec.method = getattr(nl, method)
    spec.sewi_variant = 1
    spec.nonlinearity = getattr(nl, kind)
    spec.r0 = -0.1  # quintic coefficient of the cubic-quintic kind
    _check(spec, u0, None, m, c, 1e-5 if p == nl.FP32 else 1e-9, None)


def test_kind_method_mismatch_rejected():
    import nlsb200 as nl
    from nlsb200 import workloads as W
    from nlsb200._lib import NlsError
    spec, u0, _, m, c = W.nlse_case(24, 8.0, T=0.01, nt=10, ns=2, k=8, seed=1, precision=nl.FP32)
    spec.nonlinearity = nl.NL_SINE
    with pytest.raises(NlsError) as err:
        nl.Solver(spec, u0, None, m, c)
    assert err.value.code == -1 and "nonlinearity" in str(err.value)
    spec, u0, v0, m, c = W.kg_case(24, 8.0, T=0.1, nt=10, ns=2, k=8, seed=1, precision=nl.FP32)
    spec.nonlinearity = nl.NL_SAT
    with pytest.raises(NlsError):
        nl.Solver(spec, u0, v0, m, c)
