"""Pinning against the reference's own code, compiled from its sources by
oracle/Makefile and run on the same inputs as the FP64 oracle and the engine:

  KG     device/include/kg_single.cuh step (Gautschi) / step_sv (Stormer-Verlet)
  phi^4  device/include/stochastic_phi4.cuh SP4Solver::step with its noise
         strength argument 0 (stochastic_phi4.cuh:22-24: the noise term is
         then 0 * N(0,1) = 0 at every point, so the step is deterministic;
         the reference seeds its noise from the wall clock, :25, so no run with
         noise is reproducible)
  NLSE   device/include/nlse_dev.hpp NLSESolverDevice::step (Strang SS2) and
         ::step_sewi (SEWI in the reference's operand order, a few steps: that
         order grows without bound)

with the Lanczos matrix functions (matfunc_real.hpp / lanczos.hpp,
matfunc_complex.hpp / lanczos_complex.hpp: cuBLAS, cuSPARSE, cuSOLVER syevd /
Zheevd), in 2-D and 3-D, through oracle/ref_kg.py and oracle/ref_nlse.py.

The operator reaches the reference as CSR arrays assembled from the oracle's
operator (the reference assembles it with Eigen, which is absent here; for the
NLSE class a five-member stand-in for Eigen's sparse matrix carries them); the
operator itself is pinned to the finite-volume formula in test_oracle_kat.py.
Square and cubic grids only, as the reference's solver classes.

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


# ---------------------------------------------------------------- phi^4 (noise strength 0)

def _phi4_case(prec, seed, dim):
    import nlsb200 as nl
    spec, u0, v0, m, c = _case("SP4_SV", prec, seed, dim)
    spec.rm = 0.0  # the noise strength the reference's step is given (stochastic_phi4.cuh:22-24)
    return spec, u0, v0, m, c


@pytest.mark.parametrize("dim", [2, 3])
def test_phi4_oracle_equals_reference_code(dim):
    from parity_util import run_oracle
    spec, u0, v0, m, c = _phi4_case("FP64", 71, dim)
    rt, rv, _ = run_ref(spec, u0, v0, m, 2)
    ot, ov = run_oracle(spec, u0, v0, m, c)
    assert np.all(np.isfinite(rt)) and np.abs(rt[-1] - rt[0]).max() > 1e-3
    print(f"oracle vs reference phi4 SV {dim}-D: traj {rel_l2(ot, rt):.2e} vel {rel_l2(ov, rv):.2e}")
    assert rel_l2(ot, rt) < 1e-10 and rel_l2(ov, rv) < 1e-10, (rel_l2(ot, rt), rel_l2(ov, rv))


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("prec", ["FP64", "FP32"])
def test_phi4_engine_against_reference_code(prec, dim):
    import nlsb200 as nl
    spec, u0, v0, m, c = _phi4_case(prec, 72, dim)
    rt, rv, _ = run_ref(spec, u0, v0, m, 2)
    with nl.Solver(spec, u0, v0, m, c) as s:
        s.run()
        et, ev = s.snapshots()
    tol, vtol = (1e-9, 1e-9) if prec == "FP64" else (1e-5, 1e-4)
    print(f"engine {prec} vs reference phi4 SV {dim}-D: traj {rel_l2(et, rt):.2e} vel {rel_l2(ev, rv):.2e}")
    assert rel_l2(et, rt) < tol and rel_l2(ev, rv) < vtol, (rel_l2(et, rt), rel_l2(ev, rv))


# ---------------------------------------------------------------- NLSE SS2 and SEWI

# (n, L, T, nt, ns): SS2 runs 19 steps; SEWI in the reference's order runs 4
NLSE_GRIDS = {("ss2", 2): (24, 8.0, 0.2, 20, 5), ("ss2", 3): (12, 6.0, 0.1, 10, 5),
              ("sewi", 2): (24, 8.0, 0.05, 5, 5), ("sewi", 3): (12, 6.0, 0.05, 5, 5)}


def run_ref_nlse(spec, u0, m, sewi):
    from oracle import ref_nlse
    if not ref_nlse.available():
        pytest.skip("oracle/_ref/libref_nlse.so not built (needs the reference checkout at build time)")
    return ref_nlse.run(spec, u0, m, sewi)


def _nlse_case(kind, prec, seed, dim):
    import nlsb200 as nl
    from nlsb200 import workloads as W
    n, L, T, nt, ns = NLSE_GRIDS[(kind, dim)]
    method = nl.NLSE_SEWI if kind == "sewi" else nl.NLSE_SS2
    spec, u0, _, _, c = W.nlse_case(n, L, T=T, nt=nt, ns=ns, k=12, seed=seed, dim=dim, method=method,
                                    precision=getattr(nl, prec))
    spec.sewi_variant = 0  # the reference's operand order (nlse_dev.hpp:222-225)
    m = W.mass_field(u0.shape, np.random.default_rng(seed + 1))
    return spec, u0, m, c


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("kind", ["ss2", "sewi"])
def test_nlse_oracle_equals_reference_code(kind, dim):
    from parity_util import run_oracle
    spec, u0, m, c = _nlse_case(kind, "FP64", 81, dim)
    rt, _ = run_ref_nlse(spec, u0, m, kind == "sewi")
    ot, _ = run_oracle(spec, u0, None, m, c)
    assert np.all(np.isfinite(rt)) and np.abs(rt[-1] - rt[0]).max() > 1e-3
    print(f"oracle vs reference NLSE {kind} {dim}-D: traj {rel_l2(ot, rt):.2e}")
    assert rel_l2(ot, rt) < 1e-10, rel_l2(ot, rt)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("kind", ["ss2", "sewi"])
@pytest.mark.parametrize("prec", ["FP64", "FP32"])
def test_nlse_engine_against_reference_code(kind, prec, dim):
    import nlsb200 as nl
    spec, u0, m, c = _nlse_case(kind, prec, 82, dim)
    rt, _ = run_ref_nlse(spec, u0, m, kind == "sewi")
    with nl.Solver(spec, u0, None, m, c) as s:
        s.run()
        et, _ = s.snapshots()
    tol = 1e-9 if prec == "FP64" else 1e-5
    print(f"engine {prec} vs reference NLSE {kind} {dim}-D: traj {rel_l2(et, rt):.2e}")
    assert rel_l2(et, rt) < tol, rel_l2(et, rt)
