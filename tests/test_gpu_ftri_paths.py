"""Both evaluations of f(T)e_1 in the f(T) kernel against the FP64 oracle (which
diagonalises T by QL): the Taylor series with the negative-eigenvalue
correction, taken while the argument bound (dt^2 rho for the square-root kinds
of KG, dt rho for the exponential of the NLSE; rho the Gershgorin radius of T)
is at most 4, and the QL fallback above it. On a 48^2 grid
on [-8,8]^2 (h = 0.34) the Lanczos matrices of these fields have rho of 54 to
73, so dt = 0.01 takes the first (bounds below 1) and dt = 0.6 (KG, bounds 19
to 26) or 0.3 (NLSE, bound 21) the second. This covers the cos and sinc^2
kinds (KG) and the exponential (SS2); the sinc kind of SEWI is covered by the
SEWI parity cases, whose small steps take the Taylor path.

Tolerances: rel-L2 over all snapshots, 1e-9 (FP64) and 1e-5 (FP32). The
large steps run in FP64 only: there a k-step Lanczos approximation is far from
converged (dt rho of 20), and the FP32 basis' rounding moves the result by
more than 1e-5 from the FP64 oracle's (measured 1.6e-5 for KG and 1.6e-3 for
the NLSE) whichever way f(T) is evaluated.
"""
import numpy as np
import pytest

from conftest import rel_l2
from parity_util import run_oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("method,dt,prec", [
    ("KG_GAUTSCHI", 0.01, "FP64"), ("KG_GAUTSCHI", 0.01, "FP32"), ("KG_GAUTSCHI", 0.6, "FP64"),
    ("NLSE_SS2", 0.01, "FP64"), ("NLSE_SS2", 0.01, "FP32"), ("NLSE_SS2", 0.3, "FP64")])
def test_ftri_paths(method, dt, prec):
    import nlsb200 as nl
    from nlsb200 import workloads as W
    nt, ns = 12, 3
    if method.startswith("KG"):
        spec, u0, v0, m, c = W.kg_case(48, 8.0, T=nt * dt, nt=nt, ns=ns, k=10, seed=31,
                                       method=getattr(nl, method), precision=getattr(nl, prec))
    else:
        spec, u0, v0, m, c = W.nlse_case(48, 8.0, T=nt * dt, nt=nt, ns=ns, k=12, seed=32,
                                         method=getattr(nl, method), precision=getattr(nl, prec))
    assert abs(spec.dt - dt) < 1e-15
    with nl.Solver(spec, u0, v0, m, c) as s:
        s.run()
        et, ev = s.snapshots()
    ot, ov = run_oracle(spec, u0, v0, m, c)
    tol = 1e-9 if prec == "FP64" else 1e-5
    assert np.all(np.isfinite(et))
    assert rel_l2(et, ot) < tol, rel_l2(et, ot)
    if ev is not None and ov is not None:
        assert rel_l2(ev, ov) < 10 * tol, rel_l2(ev, ov)
