"""ctypes front end of the FP64 CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline legs of ``bench.py`` as the checker / timed CPU baseline. The
product (``nlsolvers-datagen_b200``) never imports it.

The reference (konradha/nlsolvers-datagen) has no tests, golden vectors or
CPU path; the oracle restates the arithmetic of device/include/*.hpp line by
line (see oracle.cpp) and is cross-checked against dense numpy/scipy answers in
tests/test_oracle_kat.py. PINNED for the KG Gautschi and Stormer-Verlet
integrators against the reference's own device code, compiled by
oracle/Makefile into oracle/_ref (tests/test_gpu_reference_pin.py); UNPINNED
for the NLSE integrators (that code needs Eigen) and the phi^4 noise (seeded
from the wall clock).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

KG_GAUTSCHI, KG_SV, SP4_SV, SP4_GAUTSCHI, NLSE_SS2, NLSE_SEWI = range(6)
F_COS_SQRT, F_SINC2_SQRT, F_ID_SQRT, F_EXP, F_SINC = range(5)


class _Problem(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int32), ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
        ("nz", ctypes.c_int32), ("Lx", ctypes.c_double), ("Ly", ctypes.c_double),
        ("Lz", ctypes.c_double), ("T", ctypes.c_double), ("nt", ctypes.c_int32),
        ("ns", ctypes.c_int32), ("k", ctypes.c_int32), ("method", ctypes.c_int32),
        ("sewi_variant", ctypes.c_int32), ("reorth", ctypes.c_int32),
        ("max_steps", ctypes.c_int32), ("nonlinearity", ctypes.c_int32),
        ("p1", ctypes.c_double), ("q1", ctypes.c_double), ("p3", ctypes.c_double),
        ("q3", ctypes.c_double), ("rm", ctypes.c_double), ("r0", ctypes.c_double),
        ("seed", ctypes.c_uint64),
    ]


def build() -> str:
    """Compile liboracle.so with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_apply_operator.argtypes = [ctypes.c_int32] * 4 + [ctypes.c_double] * 2 + [dp, dp, dp, ctypes.c_int32]
        L.orc_tridiag_eig.argtypes = [ctypes.c_int32, dp, dp, dp, dp]
        L.orc_tridiag_eig.restype = ctypes.c_int32
        L.orc_fT_e1.argtypes = [ctypes.c_int32, dp, ctypes.c_int32, ctypes.c_int32,
                                ctypes.c_double, ctypes.c_double, dp]
        L.orc_fT_e1.restype = ctypes.c_int32
        L.orc_matfunc.argtypes = ([ctypes.c_int32] * 4 + [ctypes.c_double] * 2 + [dp] +
                                  [ctypes.c_int32] * 3 + [ctypes.c_double] * 2 +
                                  [ctypes.c_int32, dp, dp, dp])
        L.orc_matfunc.restype = ctypes.c_int32
        L.orc_philox_normal.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32]
        L.orc_philox_normal.restype = ctypes.c_double
        L.orc_run.argtypes = [ctypes.POINTER(_Problem), dp, dp, dp, dp, dp, dp]
        L.orc_run.restype = ctypes.c_int32
        L.orc_num_threads.restype = ctypes.c_int32
        L.orc_apply_bc.argtypes = [ctypes.c_int32] * 4 + [dp, ctypes.c_int32]
        L.orc_apply_bc.restype = None
        L.orc_real_begin.argtypes = [ctypes.POINTER(_Problem), dp, dp, dp, dp]
        L.orc_real_begin.restype = ctypes.c_void_p
        L.orc_real_advance.argtypes = [ctypes.c_void_p, ctypes.c_int32, dp]
        L.orc_real_advance.restype = ctypes.c_int32
        L.orc_real_end.argtypes = [ctypes.c_void_p]
        L.orc_real_end.restype = None
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _f64(a, cplx=False):
    a = np.ascontiguousarray(a, dtype=np.complex128 if cplx else np.float64)
    return a


def grid_n(dim, nx, ny, nz):
    return nx * ny * (nz if dim == 3 else 1)


def apply_operator(x, c, dim, inv_h2, sign=1.0):
    """sign * L(c) x for x shaped (ny, nx) or (nz, ny, nx)."""
    cplx = np.iscomplexobj(x)
    x = _f64(x, cplx)
    c = _f64(c)
    y = np.empty_like(x)
    nz, ny, nx = (x.shape if dim == 3 else (1,) + x.shape)
    lib().orc_apply_operator(dim, nx, ny, nz, inv_h2, sign, _p(c), _p(x.view(np.float64)),
                             _p(y.view(np.float64)), int(cplx))
    return y


def tridiag_eig(diag, sub):
    d = _f64(diag)
    e = _f64(np.concatenate([np.asarray(sub, dtype=np.float64), [0.0]]))
    n = d.size
    w = np.empty(n)
    z = np.empty(n * n)
    rc = lib().orc_tridiag_eig(n, _p(d), _p(e), _p(w), _p(z))
    if rc != 0:
        raise RuntimeError("tridiag_eig did not converge")
    return w, z.reshape(n, n).T  # columns are eigenvectors


def fT_e1(T, ftype, t):
    """f(T) e1 for a k x k Lanczos matrix (numpy (row, col) indexing)."""
    cplx = np.iscomplexobj(T) or np.iscomplexobj(t)
    Tc = _f64(np.asarray(T).T, cplx)  # column-major as the reference stores it
    k = Tc.shape[0]
    out = np.empty(k, dtype=np.complex128 if cplx else np.float64)
    t = complex(t)
    rc = lib().orc_fT_e1(k, _p(Tc.view(np.float64)), int(cplx), ftype, t.real, t.imag,
                         _p(out.view(np.float64)))
    if rc != 0:
        raise RuntimeError("fT_e1 failed")
    return out


def matfunc(x, c, dim, inv_h2, sign, k, ftype, t, reorth=True):
    """beta0 V f(T) e1 (the reference's MatrixFunctionApplicator::apply); returns (y, T)."""
    cplx = np.iscomplexobj(x) or ftype in (F_EXP, F_SINC)
    x = _f64(x, cplx)
    c = _f64(c)
    y = np.empty_like(x)
    Tm = np.empty(k * k, dtype=np.complex128 if cplx else np.float64)
    nz, ny, nx = (x.shape if dim == 3 else (1,) + x.shape)
    t = complex(t)
    rc = lib().orc_matfunc(dim, nx, ny, nz, inv_h2, sign, _p(c), k, int(cplx), ftype, t.real,
                           t.imag, int(reorth), _p(x.view(np.float64)), _p(y.view(np.float64)),
                           _p(Tm.view(np.float64)))
    if rc != 0:
        raise RuntimeError(f"matfunc failed: {rc}")
    return y, Tm.reshape(k, k).T


def apply_bc(u, dim):
    """The reference's ghost copies on a copy of u ((ny, nx) or (nz, ny, nx))."""
    cplx = np.iscomplexobj(u)
    u = _f64(u, cplx).copy()
    nz, ny, nx = (u.shape if dim == 3 else (1,) + u.shape)
    lib().orc_apply_bc(dim, nx, ny, nz, _p(u.view(np.float64)), int(cplx))
    return u


def philox_normal(seed, step, point):
    return lib().orc_philox_normal(seed, step, point)


@dataclass
class Problem:
    """Mirror of orc_problem; sizes include the ghost ring as the drivers' argv."""
    dim: int
    nx: int
    ny: int
    nz: int = 1
    Lx: float = 10.0
    Ly: float = 10.0
    Lz: float = 10.0
    T: float = 1.0
    nt: int = 100
    ns: int = 10
    k: int = 10
    method: int = KG_GAUTSCHI
    sewi_variant: int = 0
    reorth: int = 1
    max_steps: int = 0
    p1: float = 0.0
    q1: float = 0.0
    p3: float = -1.0
    q3: float = 0.0
    rm: float = 0.0
    r0: float = 0.0
    seed: int = 0
    nonlinearity: int = 0
    extra: dict = field(default_factory=dict)

    def struct(self):
        s = _Problem()
        for name, _ in _Problem._fields_:
            setattr(s, name, getattr(self, name))
        return s


def reference_coefficients(method, dim, nx, Lx, dt):
    """The reference's equation coefficients and default Krylov dimension per
    executable, written out here from its sources (not taken from the
    product library) so that a wrong default in the product cannot pass
    unseen:
      KG Gautschi / SV: g(u) = -m u^3               (kg_single.cuh:105-108, :152-155)
      phi^4 SV:         g(u) = -m (u - u^3 + s xi)  (stochastic_phi4.cuh:52),
                        s = 0.01 sqrt(2 dx) / dt    (stochastic_phi4_dev.hpp:47-51)
      NLSE:             rho = m |u|^2               (nlse_dev.hpp:20-29)
      k: KG / phi^4 10 (kg_driver_dev_2d.cpp:138, sp4_sv_driver_dev_2d.cpp:135),
         SS2 2-D 20 / 3-D 25 (nlse_cubic_driver_2d.cpp:104, nlse_cubic_driver_3d.cpp:112),
         SEWI 2-D 10 / 3-D 15 (nlse_cubic_sewi_driver_2d.cpp:104, _3d.cpp:112).
    In the oracle's form g(u) = (p1 m + q1) u + (p3 m + q3) u^3 + (rm m + r0) xi."""
    c = dict(p1=0.0, q1=0.0, p3=0.0, q3=0.0, rm=0.0, r0=0.0, nonlinearity=0)
    if method in (KG_GAUTSCHI, KG_SV):
        c.update(p3=-1.0, k=10)
    elif method in (SP4_SV, SP4_GAUTSCHI):
        dx = 2.0 * Lx / (nx - 1)
        c.update(p1=-1.0, p3=1.0, rm=-(0.01 * np.sqrt(2.0 * dx) / dt), k=10)
    elif method == NLSE_SS2:
        c.update(p3=1.0, k=20 if dim == 2 else 25)
    elif method == NLSE_SEWI:
        c.update(p3=1.0, k=10 if dim == 2 else 15)
    else:
        raise ValueError(f"unknown method {method}")
    return c


def run(prob: Problem, u0, v0, m, c):
    """Full driver run; returns (traj, vel) shaped (ns, *grid) (vel None for NLSE)."""
    cplx = prob.method in (NLSE_SS2, NLSE_SEWI)
    shape = (prob.nz, prob.ny, prob.nx) if prob.dim == 3 else (prob.ny, prob.nx)
    u0 = _f64(np.reshape(u0, shape), cplx)
    v0 = _f64(np.zeros(shape) if v0 is None else np.reshape(v0, shape))
    m = _f64(np.reshape(m, shape))
    c = _f64(np.reshape(c, shape))
    traj = np.zeros((prob.ns,) + shape, dtype=np.complex128 if cplx else np.float64)
    vel = np.zeros((prob.ns,) + shape)
    s = prob.struct()
    rc = lib().orc_run(ctypes.byref(s), _p(u0.view(np.float64)), _p(v0), _p(m), _p(c),
                       _p(traj.view(np.float64)), _p(vel))
    if rc != 0:
        raise RuntimeError(f"oracle run failed: {rc}")
    return traj, (None if cplx else vel)


class RealStepper:
    """Stateful KG / phi4 oracle trajectory (pure step timing)."""

    def __init__(self, prob: Problem, u0, v0, m, c):
        shape = (prob.nz, prob.ny, prob.nx) if prob.dim == 3 else (prob.ny, prob.nx)
        self._arrs = [_f64(np.reshape(a, shape)) for a in
                      (u0, np.zeros(shape) if v0 is None else v0, m, c)]
        self._s = prob.struct()
        self._h = lib().orc_real_begin(ctypes.byref(self._s), *[_p(a) for a in self._arrs])
        if not self._h:
            raise RuntimeError("orc_real_begin failed")
        self.shape = shape

    def advance(self, nsteps, want_u=False):
        u = np.empty(self.shape) if want_u else None
        rc = lib().orc_real_advance(self._h, nsteps, _p(u) if want_u else None)
        if rc != 0:
            raise RuntimeError(f"oracle advance failed: {rc}")
        return u

    def close(self):
        if self._h:
            lib().orc_real_end(self._h)
            self._h = None

    def __del__(self):
        self.close()


def num_threads():
    return lib().orc_num_threads()
