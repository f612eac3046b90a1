"""Pinning against the reference's own code: the reference's KG device
solver (device/include/kg_single.cuh step / step_sv with the Lanczos matrix
functions of matfunc_real.hpp and lanczos.hpp, the SpMV of spmv.hpp and the
ghost copies of boundaries.cuh, 2-D and 3-D), compiled from its sources into
oracle/_ref/libref_kg.so by oracle/Makefile, is run on the same inputs as the
FP64 oracle and the engine.

The operator reaches the reference as CSR arrays assembled from the oracle's
operator (the reference assembles it with Eigen, which is absent here); the
operator itself is pinned to the finite-volume formula in test_oracle_kat.py.
Square and cubic grids only, as the reference's solver class (kg_dev.hpp:38-45).

Tolerances (rel-L2 over all snapshots): oracle 1e-10 and FP64 engine 1e-9
(FP64 arithmetic in different summation orders; the engine has no
re-orthogonalisation pass), FP32 engine 1e-5 (velocity 1e-4).
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libref_kg.so")


def _ref_lib():
    if not os.path.exists(REF_LIB):
        pytest.skip("oracle/_ref/libref_kg.so not built (needs the reference checkout at build time)")
    L = ctypes.CDLL(REF_LIB)
    ip, dp = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double)
    i32 = ctypes.c_int32
    L.ref_kg_run.argtypes = [i32, i32, i32, ip, ip, dp, i32, i32, dp, dp, dp, ctypes.c_double, i32, i32, dp, dp,
                             dp]
    L.ref_kg_run.restype = ctypes.c_int
    return L


def _csr(spec, sign):
    """CSR (int32, sorted columns) of sign * L on the full grid, assembled from
    the oracle's operator applied to probe vectors: a point couples only to the
    points within one cell of it, so the points of one colour of a 3-colouring
    per axis have disjoint supports and one probe per colour gives all their
    columns. Checked for symmetry and consistency before it reaches the
    reference's device code."""
    import itertools
    from oracle import oracle as O
    shape = spec.shape
    n = int(np.prod(shape))
    dx = 2 * spec.Lx / (spec.nx - 1)
    inv_h2 = 1.0 / (dx * (2 * spec.Ly / (spec.ny - 1))) if spec.dim == 2 else 1.0 / (dx * dx)
    c = np.ones(shape)
    idx = np.indices(shape).reshape(len(shape), -1)
    colour = sum(idx[a] % 3 * 3 ** a for a in range(len(shape)))
    rows, cols, vals = [], [], []
    for col in range(3 ** len(shape)):
        pts = idx[:, colour == col]
        probe = np.zeros(shape)
        probe[tuple(pts)] = 1.0
        y = O.apply_operator(probe, c, spec.dim, inv_h2, sign)
        for off in itertools.product((-1, 0, 1), repeat=len(shape)):
            q = pts + np.array(off)[:, None]
            ok = np.all((q >= 0) & (q < np.array(shape)[:, None]), axis=0)
            v = y[tuple(q[:, ok])]
            nz = v != 0
            rows.append(np.ravel_multi_index(tuple(q[:, ok][:, nz]), shape))
            cols.append(np.ravel_multi_index(tuple(pts[:, ok][:, nz]), shape))
            vals.append(v[nz])
    rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    t = np.lexsort((rows, cols))  # the transpose's entries in row-major order
    assert np.array_equal(cols[t], rows) and np.array_equal(rows[t], cols) and np.array_equal(vals[t], vals)
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(indptr, rows + 1, 1)
    indptr = np.cumsum(indptr).astype(np.int32)
    indices = cols.astype(np.int32)
    assert indptr[0] == 0 and indptr[-1] == len(indices) and np.all(np.diff(indptr) >= 0)
    assert indices.min() >= 0 and indices.max() < n
    return indptr, indices, vals.astype(np.float64)


def run_ref(spec, u0, v0, m, method):
    """The reference's code on one trajectory: (traj, vel, step-loop ms)."""
    L = _ref_lib()
    indptr, indices, vals = _csr(spec, -1.0 if method == 0 else 1.0)
    traj = np.zeros((spec.ns,) + spec.shape)
    vel = np.zeros((spec.ns,) + spec.shape)
    args = [np.ascontiguousarray(a, dtype=np.float64) for a in (u0, v0, m)]
    pi = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    pd = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    ms = ctypes.c_double(0.0)
    rc = L.ref_kg_run(spec.dim, method, spec.nx, pi(indptr), pi(indices), pd(vals), len(vals), spec.k, pd(args[0]),
                      pd(args[1]), pd(args[2]), spec.dt, spec.nt, spec.ns, pd(traj), pd(vel), ctypes.byref(ms))
    assert rc == 0, rc
    return traj, vel, ms.value


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
