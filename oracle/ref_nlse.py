"""ctypes front end of oracle/_ref/libref_nlse.so: the reference's own NLSE
device code (device/include/nlse_dev.hpp NLSESolverDevice step = Strang SS2
and step_sewi = SEWI, with the complex Lanczos matrix functions of
matfunc_complex.hpp and lanczos_complex.hpp and the ghost copies of
boundaries.cuh), compiled from its sources by oracle/Makefile with the driver
oracle/ref/ref_nlse.cu and the Eigen sparse-matrix stand-in
oracle/ref/eigen_stub.

TEST INFRASTRUCTURE ONLY: used by tests/ to pin the oracle and the engine to
the reference's code. The product never loads it. The library exists only
where the reference checkout was present at build time; `available()` says
whether it was built.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from oracle import ref_kg

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libref_nlse.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        ip, dp, i32 = ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double), ctypes.c_int32
        L.ref_nlse_run.argtypes = [i32, i32, i32, ip, ip, dp, i32, i32, dp, dp, ctypes.c_double, i32, i32, dp, dp]
        L.ref_nlse_run.restype = ctypes.c_int
        _lib = L
    return _lib


def run(spec, u0, m, sewi):
    """One NLSE trajectory through the reference's code (sewi 0: step, the
    Strang SS2 of nlse_dev.hpp:187-203; 1: step_sewi, nlse_dev.hpp:205-239,
    the reference's own operand order): (traj (ns, ...) complex128, step-loop
    ms). The operator is L itself (nlse_cubic_driver_2d.cpp:94-97), here as
    complex CSR with real values. Square and cubic grids only, as the class
    (nlse_dev.hpp:133-140)."""
    L = lib()
    indptr, indices, vals = ref_kg.csr(spec, 1.0)
    cvals = np.ascontiguousarray(vals.astype(np.complex128))
    u = np.ascontiguousarray(u0, dtype=np.complex128)
    mm = np.ascontiguousarray(m, dtype=np.float64)
    traj = np.zeros((spec.ns,) + spec.shape, dtype=np.complex128)
    pi = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    pd = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    ms = ctypes.c_double(0.0)
    rc = L.ref_nlse_run(spec.dim, int(sewi), spec.nx, pi(indptr), pi(indices), pd(cvals.view(np.float64)),
                        len(vals), spec.k, pd(u.view(np.float64)), pd(mm), spec.dt, spec.nt, spec.ns,
                        pd(traj.view(np.float64)), ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference NLSE run failed: {rc}")
    return traj, ms.value
