"""Pinning against the reference's own code: the reference's KG device
solver (device/include/kg_single.cuh step / step_sv with the Lanczos matrix
functions of matfunc_real.hpp and lanczos.hpp, the SpMV of spmv.hpp and the
ghost copies of boundaries.cuh, 2-D and 3-D), compiled from its sources into
oracle/_ref/libref_kg.so by oracle/Makefile and driven through oracle/ref_kg.py,
is run on the same inputs as the FP64 oracle and the engine.

The operator reaches the reference as CSR arrays assembled from the oracle's
operator (the reference assembles it with Eigen, which is absent here); the
operator itself is pinned to the finite-volume formula in test_oracle_kat.py.
Square and cubic grids only, as the reference's solver class (kg_dev.hpp:38-45).

Tolerances (rel-L2 over all snapshots): oracle 1e-10 and FP64 engine 1e-9
(FP64 arithmetic in different summation orders; the engine has no
re-orthogonalisation pass), FP32 engine 1e-5 (velocity 1e-4).
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def run_ref(spec, u0, v0, m, method):
    """The reference's code on one trajectory: (traj, vel, step-loop ms)."""
    from oracle import ref_kg
    if not ref_kg.available():
        pytest.skip("oracle/_ref/libref_kg.so not built (needs the reference checkout at build time)")
    return ref_kg.run(spec, u0, v0, m, method)


# (dim, n, L, T, nt, ns): a 24^2 square and a 12^3 cube
GRIDS = {2: (24, 8.0, 0.5, 50, 5), 3: (12, 6.0, 0.3, 30, 3)}


def _case(method_name, prec, seed, dim):
    import nlsb200 as nl
    from nlsb200 import workloads as W
    n, L, T, nt, ns = GRIDS[dim]
    spec, u0, v0, m, c = W.kg_case(n, L, T=T, nt=nt, ns=ns, k=10, seed=seed, dim=dim,
                                   method=getattr(nl, method_name), precision=getattr(nl, prec))
    v0 = 0.2 * np.random.default_rng(seed).standard_normal(u0.shape)
    return spec, u0, v0, m, c


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("method_name,method", [("KG_GAUTSCHI", 0), ("KG_SV", 1)])
def test_oracle_equals_reference_code(method_name, method, dim):
    from parity_util import run_oracle
    spec, u0, v0, m, c = _case(method_name, "FP64", 61, dim)
    rt, rv, _ = run_ref(spec, u0, v0, m, method)
    ot, ov = run_oracle(spec, u0, v0, m, c)
    assert np.all(np.isfinite(rt)) and np.abs(rt[-1] - rt[0]).max() > 1e-3  # the field moved
    print(f"oracle vs reference {method_name} {dim}-D: traj {rel_l2(ot, rt):.2e} vel {rel_l2(ov, rv):.2e}")
    assert rel_l2(ot, rt) < 1e-10 and rel_l2(ov, rv) < 1e-10, (rel_l2(ot, rt), rel_l2(ov, rv))


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("method_name,method", [("KG_GAUTSCHI", 0), ("KG_SV", 1)])
@pytest.mark.parametrize("prec", ["FP64", "FP32"])
def test_engine_against_reference_code(method_name, method, prec, dim):
    import nlsb200 as nl
    spec, u0, v0, m, c = _case(method_name, prec, 62, dim)
    rt, rv, _ = run_ref(spec, u0, v0, m, method)
    with nl.Solver(spec, u0, v0, m, c) as s:
        s.run()
        et, ev = s.snapshots()
    tol, vtol = (1e-9, 1e-9) if prec == "FP64" else (1e-5, 1e-4)
    print(f"engine {prec} vs reference {method_name} {dim}-D: traj {rel_l2(et, rt):.2e} vel {rel_l2(ev, rv):.2e}")
    assert rel_l2(et, rt) < tol and rel_l2(ev, rv) < vtol, (rel_l2(et, rt), rel_l2(ev, rv))
