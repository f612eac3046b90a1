"""ctypes front end of oracle/_ref/libref_kg.so: the reference's own KG and
phi^4 device code (device/include/kg_single.cuh step / step_sv and
stochastic_phi4.cuh SP4Solver::step, with the Lanczos matrix functions of
matfunc_real.hpp and lanczos.hpp, the SpMV of spmv.hpp and the ghost copies of
boundaries.cuh), compiled from its sources by oracle/Makefile with the driver
oracle/ref/ref_kg.cu.

TEST INFRASTRUCTURE ONLY: used by tests/ (to pin the oracle and the engine to
the reference's code) and by bench.py's reference arm (to time the reference's
own per-trajectory GPU path beside the CPU baseline). The product never loads
it. The library exists only where the reference checkout was present at build
time; `available()` says whether it was built.
"""
from __future__ import annotations

import ctypes
import itertools
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libref_kg.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        ip, dp, i32 = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double), ctypes.c_int32
        L.ref_kg_run.argtypes = [i32, i32, i32, ip, ip, dp, i32, i32, dp, dp, dp, ctypes.c_double, i32, i32,
                                 dp, dp, dp, ctypes.c_double]
        L.ref_kg_run.restype = ctypes.c_int
        _lib = L
    return _lib


def csr(spec, sign):
    """CSR (int32, sorted columns) of sign * L on the full grid, assembled from
    the oracle's operator applied to probe vectors: a point couples only to the
    points within one cell of it, so the points of one colour of a 3-colouring
    per axis have disjoint supports and one probe per colour gives all their
    columns. Checked for symmetry and consistency before it reaches the
    reference's device code (the reference assembles it with Eigen,
    laplacians.hpp, which is absent here)."""
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


def run(spec, u0, v0, m, method, sp4_scale=0.0):
    """One trajectory through the reference's code (method 0: Gautschi with
    A = -L, 1: Stormer-Verlet with L, 2: the phi^4 step with L and noise
    strength sp4_scale, stochastic_phi4.cuh:19-77): (traj, vel, step-loop ms).
    Square and cubic grids only, as the reference's solver classes
    (kg_dev.hpp:38-45, stochastic_phi4_dev.hpp:37-44)."""
    L = lib()
    indptr, indices, vals = csr(spec, -1.0 if method == 0 else 1.0)
    traj = np.zeros((spec.ns,) + spec.shape)
    vel = np.zeros((spec.ns,) + spec.shape)
    args = [np.ascontiguousarray(a, dtype=np.float64) for a in (u0, v0, m)]
    pi = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    pd = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    ms = ctypes.c_double(0.0)
    rc = L.ref_kg_run(spec.dim, method, spec.nx, pi(indptr), pi(indices), pd(vals), len(vals), spec.k,
                      pd(args[0]), pd(args[1]), pd(args[2]), spec.dt, spec.nt, spec.ns, pd(traj), pd(vel),
                      ctypes.byref(ms), float(sp4_scale))
    if rc != 0:
        raise RuntimeError(f"reference KG run failed: {rc}")
    return traj, vel, ms.value
