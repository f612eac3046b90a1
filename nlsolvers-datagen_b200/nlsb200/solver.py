"""Python mirror of the reference's solver interface, over the C ABI.

``Solver`` replaces one reference solver object plus its driver loop
(``KGESolverDevice`` kg_dev.hpp:32-131, ``SP4SolverDevice``
stochastic_phi4_dev.hpp:29-33, ``NLSESolverDevice`` nlse_dev.hpp:78-335, loop
kg_driver_dev_2d.cpp:144-153). ``Pool`` is the batched / continuous-batching
engine many trajectories share.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import (FP32, FP64, KG_GAUTSCHI, KG_SV, NL_CQ, NL_DSINE, NL_POLY, NL_SAT, NL_SINE, NL_SINH,
                   NLSE_SEWI, NLSE_SS2, SP4_GAUTSCHI, SP4_SV, NlsError, check, lib)

COMPLEX_METHODS = (NLSE_SS2, NLSE_SEWI)
KRYLOV_METHODS = (KG_GAUTSCHI, SP4_GAUTSCHI, NLSE_SS2, NLSE_SEWI)


@dataclass
class Spec:
    """Problem description; grid sizes include the ghost ring (driver argv)."""
    method: int
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
    k: int | None = None
    precision: int = FP32
    sewi_variant: int = 0
    p1: float | None = None
    q1: float = 0.0
    p3: float | None = None
    q3: float = 0.0
    rm: float | None = None
    r0: float = 0.0
    seed: int = 0
    nonlinearity: int = 0   # NL_* kind (0: the reference's polynomial / cubic form)

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx) if self.dim == 3 else (self.ny, self.nx)

    @property
    def n(self):
        return int(np.prod(self.shape))

    @property
    def dt(self):
        return self.T / self.nt

    @property
    def complex(self):
        return self.method in COMPLEX_METHODS

    def struct(self, has_c: bool) -> _lib.Problem:
        p = _lib.Problem()
        check(lib().nls_problem_defaults(ctypes.byref(p), self.method, self.dim))
        p.nx, p.ny, p.nz = self.nx, self.ny, (self.nz if self.dim == 3 else 1)
        p.Lx, p.Ly, p.Lz = self.Lx, self.Ly, self.Lz
        p.T, p.nt, p.ns = self.T, self.nt, self.ns
        if self.k is not None:
            p.k = self.k
        p.precision = self.precision
        p.sewi_variant = self.sewi_variant
        p.has_c = 1 if has_c else 0
        if self.p1 is not None:
            p.p1 = self.p1
        if self.p3 is not None:
            p.p3 = self.p3
        p.q1, p.q3, p.r0 = self.q1, self.q3, self.r0
        if self.rm is not None:
            p.rm = self.rm
        elif self.method in (SP4_SV, SP4_GAUTSCHI):
            p.rm = reference_phi4_rm(self)
        p.seed = self.seed
        p.nonlinearity = self.nonlinearity
        return p


def reference_phi4_rm(spec: Spec) -> float:
    """-alpha sqrt(kBT dx)/dt with alpha = 0.01, kBT = 2, dx = 2L/(nx-1)
    (stochastic_phi4_dev.hpp:47-51): the noise enters as -m s xi."""
    dx = 2 * spec.Lx / (spec.nx - 1)
    return -(0.01 * math.sqrt(2.0 * dx) / spec.dt)


def pinned_empty(shape, dtype=np.float64):
    """numpy array in page-locked host memory (freed with the array)."""
    import weakref
    dt = np.dtype(dtype)
    nbytes = int(np.prod(shape)) * dt.itemsize
    ptr = ctypes.c_void_p()
    check(lib().nls_host_alloc(max(nbytes, 1), ctypes.byref(ptr)))
    buf = (ctypes.c_char * max(nbytes, 1)).from_address(ptr.value)
    weakref.finalize(buf, lib().nls_host_free, ctypes.c_void_p(ptr.value))
    return np.frombuffer(buf, dtype=dt, count=int(np.prod(shape))).reshape(shape)


def _downsample(u, target_shape, L):
    u = np.asarray(u)
    cplx = np.iscomplexobj(u)
    dim = u.ndim - 1
    tgt = tuple(int(t) for t in target_shape)
    src = np.ascontiguousarray(u, dtype=np.complex128 if cplx else np.float64)
    out = np.empty((u.shape[0],) + tgt, dtype=src.dtype)
    shape = (ctypes.c_int64 * 3)(*u.shape[1:])
    tg = (ctypes.c_int64 * 3)(*tgt)
    hw = (ctypes.c_double * 3)(*[float(x) for x in L])
    check(lib().nls_downsample_linear(dim, shape, tg, hw, u.shape[0], int(cplx), _dptr(src.view(np.float64)),
                                      _dptr(out.view(np.float64))))
    return out.astype(u.dtype)


def downsample_interpolation(u, target_shape, Lx, Ly):
    """Drop-in for the reference's downsample_interpolation
    (scripts/downsampling.py:68-103): u (frames, n0, n1) onto linspace grids of
    target_shape, computed on the GPU; equal to it bitwise."""
    assert np.ndim(u) == 3 and len(target_shape) == 2
    return _downsample(u, target_shape, (Lx, Ly))


def downsample_interpolation_3d(u, target_shape, Lx, Ly, Lz):
    """Drop-in for the reference's downsample_interpolation_3d
    (scripts/downsampling.py:215-257): u (frames, n0, n1, n2)."""
    assert np.ndim(u) == 4 and len(target_shape) == 3
    return _downsample(u, target_shape, (Lx, Ly, Lz))


def _downsample_fft(u, target_shape):
    u = np.asarray(u)
    cplx = np.iscomplexobj(u)
    dim = u.ndim - 1
    tgt = tuple(int(t) for t in target_shape)
    if len(tgt) != dim:
        raise ValueError(f"target shape {tgt} does not match {dim}-D frames")
    src = np.ascontiguousarray(u, dtype=np.complex128 if cplx else np.float64)
    out = np.empty((u.shape[0],) + tgt, dtype=src.dtype)
    shape = (ctypes.c_int64 * 3)(*u.shape[1:])
    tg = (ctypes.c_int64 * 3)(*tgt)
    check(lib().nls_downsample_fft(dim, shape, tg, u.shape[0], int(cplx), _dptr(src.view(np.float64)),
                                   _dptr(out.view(np.float64))))
    return out.astype(u.dtype)


def downsample_fft(u, target_shape):
    """Drop-in for the reference's downsample_fft (scripts/downsampling.py:10-35):
    u (frames, n0, n1), centred crop of the orthonormal spectrum to
    target_shape, computed on the GPU in FP64."""
    assert np.ndim(u) == 3 and len(target_shape) == 2
    return _downsample_fft(u, target_shape)


def downsample_fft_3d(u, target_shape):
    """Drop-in for the reference's downsample_fft_3d
    (scripts/downsampling.py:147-178): u (frames, n0, n1, n2)."""
    assert np.ndim(u) == 4 and len(target_shape) == 3
    return _downsample_fft(u, target_shape)


def _dptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _prep(spec: Spec, u0, v0, m, c):
    shape = spec.shape
    u0 = np.ascontiguousarray(np.reshape(u0, shape),
                              dtype=np.complex128 if spec.complex else np.float64)
    v0 = None if (v0 is None or spec.complex) else np.ascontiguousarray(np.reshape(v0, shape), dtype=np.float64)
    m = np.ascontiguousarray(np.reshape(m, shape), dtype=np.float64)
    has_c = c is not None and not np.all(np.asarray(c) == 1.0)
    c = np.ascontiguousarray(np.reshape(c, shape), dtype=np.float64) if has_c else None
    return u0, v0, m, c, has_c


class Solver:
    """One trajectory on the GPU: snapshot 0 is the input; ``run()`` executes
    the driver loop i = 1..nt-1; ``snapshots()`` returns (traj, vel)."""

    def __init__(self, spec: Spec, u0, v0, m, c=None):
        self.spec = spec
        u0, v0, m, c, has_c = _prep(spec, u0, v0, m, c)
        self._keep = (u0, v0, m, c)
        self._h = ctypes.c_void_p()
        check(lib().nls_create(ctypes.byref(spec.struct(has_c)), _dptr(u0.view(np.float64)),
                               _dptr(v0), _dptr(m), _dptr(c), ctypes.byref(self._h)))

    def step(self, nsteps: int = 1):
        check(lib().nls_step(self._h, nsteps))

    def run(self):
        check(lib().nls_run(self._h))

    def enable_diagnostics(self):
        """Per-snapshot energy / mass (ns x 4, filled as snapshots complete;
        see nls_pool_set_diagnostics). Call before the first step."""
        self._diag = np.zeros((self.spec.ns, 4))
        check(lib().nls_set_diagnostics(self._h, _dptr(self._diag)))
        return self._diag

    def diagnostics(self):
        """The diagnostics array after waiting for all snapshots."""
        self.snapshots()
        return self._diag

    def steps_done(self) -> int:
        v = ctypes.c_int32()
        check(lib().nls_steps_done(self._h, ctypes.byref(v)))
        return v.value

    def snapshots(self):
        s = self.spec
        traj = np.zeros((s.ns,) + s.shape, dtype=np.complex128 if s.complex else np.float64)
        vel = None if s.complex else np.zeros((s.ns,) + s.shape)
        check(lib().nls_snapshot(self._h, _dptr(traj.view(np.float64)), _dptr(vel)))
        return traj, vel

    def close(self):
        if self._h:
            lib().nls_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


@dataclass
class SlotInfo:
    slot: int
    spec: Spec
    traj: np.ndarray
    vel: np.ndarray | None
    inputs: tuple = field(default_factory=tuple)
    diag: np.ndarray | None = None
    ds_traj: np.ndarray | None = None   # downsampled snapshots (set_downsample)
    ds_vel: np.ndarray | None = None
    out_npy: tuple | None = None        # (traj path, vel path or None): snapshots streamed to .npy
    streams: list | None = None         # [(memmap, source array)] once streaming started
    written: int = 0                    # snapshots already in the files


class Pool:
    """Batched engine: trajectories of one (method, dim, k, precision) with any
    grid sizes step together; admit/release between steps."""

    def __init__(self, method: int, dim: int, k: int | None, precision: int,
                 capacity_points: int, max_slots: int, graphs: bool = True,
                 segment: int | None = None, final_segment: int | None = None):
        if k is None:
            p = _lib.Problem()
            check(lib().nls_problem_defaults(ctypes.byref(p), method, dim))
            k = p.k
        self.method, self.dim, self.k, self.precision = method, dim, k, precision
        self._p = ctypes.c_void_p()
        check(lib().nls_pool_create(method, dim, k, precision, int(capacity_points),
                                    int(max_slots), ctypes.byref(self._p)))
        self.slots: dict[int, SlotInfo] = {}
        if not graphs:
            check(lib().nls_pool_set_graphs(self._p, 0))
        if segment:
            check(lib().nls_pool_set_segment(self._p, int(segment)))
        if final_segment:
            check(lib().nls_pool_set_final_segment(self._p, int(final_segment)))

    def admit(self, spec: Spec, u0, v0, m, c=None, traj=None, vel=None, out_npy=None):
        """Returns the slot id, or None when the pool is full right now.

        out_npy = (traj_path, vel_path or None): the snapshots are also written
        to these .npy files (the reference drivers' layout: (ns, ny, nx) or
        (ns, nz, ny, nx), '<f8' or '<c16') as they reach the host, by poll(),
        stream() and release()."""
        u0, v0, m, c, has_c = _prep(spec, u0, v0, m, c)
        dt = np.complex128 if spec.complex else np.float64
        if traj is None:
            traj = pinned_empty((spec.ns,) + spec.shape, dt) if out_npy else np.zeros((spec.ns,) + spec.shape, dtype=dt)
        if vel is None and not spec.complex:
            vel = pinned_empty((spec.ns,) + spec.shape) if out_npy else np.zeros((spec.ns,) + spec.shape)
        slot = ctypes.c_int32(-1)
        rc = lib().nls_pool_admit(self._p, ctypes.byref(spec.struct(has_c)),
                                  _dptr(u0.view(np.float64)), _dptr(v0), _dptr(m), _dptr(c),
                                  _dptr(traj.view(np.float64)), _dptr(vel), ctypes.byref(slot))
        if rc == _lib.NLS_ERR_CAPACITY:
            return None
        check(rc)
        self.slots[slot.value] = SlotInfo(slot.value, spec, traj, vel, (u0, v0, m, c),
                                          out_npy=tuple(out_npy) if out_npy else None)
        return slot.value

    def stream(self, slot: int) -> int:
        """Write the snapshots that reached the host since the last call to the
        slot's .npy files (admit's out_npy); returns how many are complete."""
        info = self.slots[slot]
        n = ctypes.c_int32()
        check(lib().nls_pool_snapshots_ready(self._p, slot, ctypes.byref(n)))
        if info.out_npy:
            self._write_frames(info, n.value)
        return n.value

    @staticmethod
    def _write_frames(info, ready):
        if info.streams is None:
            src = [info.ds_traj if info.ds_traj is not None else info.traj,
                   info.ds_vel if info.ds_traj is not None else info.vel]
            info.streams = []
            for path, a in zip(info.out_npy, src):
                if path is not None and a is not None:
                    mm = np.lib.format.open_memmap(path, mode="w+", dtype=a.dtype, shape=a.shape)
                    info.streams.append((mm, a))
        if ready > info.written:
            for mm, a in info.streams:
                mm[info.written:ready] = a[info.written:ready]
                mm.flush()
            info.written = ready

    def enable_diagnostics(self, slot: int):
        """Per-snapshot energy / mass of `slot` (ns x 4; see
        nls_pool_set_diagnostics); call before the slot's first step."""
        info = self.slots[slot]
        info.diag = np.zeros((info.spec.ns, 4))
        check(lib().nls_pool_set_diagnostics(self._p, slot, _dptr(info.diag)))
        return info.diag

    def set_downsample(self, slot: int, target_shape, mode: str = "linear"):
        """Downsample every snapshot of `slot` on the device to `target_shape`
        (array-axis order) before its copy to the host, as the reference's HDF5
        aggregation does on the host (see nls_pool_set_downsample). Call before
        the slot's first step; returns (ds_traj, ds_vel) of shape
        (ns,) + target_shape, filled as snapshots complete (ds_vel is None for
        the NLSE); the slot's full-size outputs then hold snapshot 0 only.
        mode "linear": linear interpolation (nls_pool_set_downsample); "fft":
        the spectral crop (nls_pool_set_downsample_fft)."""
        if mode not in ("linear", "fft"):
            raise ValueError(f"unknown downsampling mode {mode!r}")
        info = self.slots[slot]
        spec = info.spec
        tgt = tuple(int(t) for t in target_shape)
        if len(tgt) != spec.dim:
            raise ValueError(f"target shape {tgt} does not match a {spec.dim}-D slot")
        traj = np.zeros((spec.ns,) + tgt, dtype=np.complex128 if spec.complex else np.float64)
        vel = None if spec.complex else np.zeros((spec.ns,) + tgt)
        t32 = (ctypes.c_int32 * 3)(*(tgt + (1,) * (3 - len(tgt))))
        fn = lib().nls_pool_set_downsample_fft if mode == "fft" else lib().nls_pool_set_downsample
        check(fn(self._p, slot, t32, _dptr(traj.view(np.float64)), _dptr(vel)))
        info.ds_traj, info.ds_vel = traj, vel
        return traj, vel

    def step(self, nsteps: int = 1):
        check(lib().nls_pool_step(self._p, int(nsteps)))

    def step_timed(self, nsteps: int) -> float:
        """Advance nsteps steps; device time in ms (CUDA events on the pool stream)."""
        ms = ctypes.c_float()
        check(lib().nls_pool_step_timed(self._p, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def poll(self, slot: int):
        done, fin = ctypes.c_int32(), ctypes.c_int32()
        check(lib().nls_pool_poll(self._p, slot, ctypes.byref(done), ctypes.byref(fin)))
        if self.slots[slot].out_npy:
            self.stream(slot)
        return done.value, bool(fin.value)

    def release(self, slot: int) -> SlotInfo:
        check(lib().nls_pool_release(self._p, slot))
        info = self.slots.pop(slot)
        if info.out_npy:
            self._write_frames(info, info.spec.ns)  # every copy completed in release
            info.streams = None  # closes the memmaps
        return info

    def sync(self):
        check(lib().nls_pool_sync(self._p))

    def usage(self):
        occ, free = ctypes.c_int32(), ctypes.c_int64()
        check(lib().nls_pool_usage(self._p, ctypes.byref(occ), ctypes.byref(free)))
        return occ.value, free.value

    def time_pass(self, j: int, iters: int):
        ms, pts = ctypes.c_float(), ctypes.c_int64()
        check(lib().nls_pool_time_pass(self._p, j, iters, ctypes.byref(ms), ctypes.byref(pts)))
        return ms.value, pts.value

    def fence(self) -> int:
        """Ticket of the device work queued so far (steps and admissions)."""
        t = ctypes.c_int32()
        check(lib().nls_pool_fence(self._p, ctypes.byref(t)))
        return t.value

    def fence_wait(self, ticket: int):
        """Block until the work before fence `ticket` has run; raises on a
        slot's device-side failure as sync() does."""
        check(lib().nls_pool_fence_wait(self._p, ticket))

    def set_priority(self, high: bool):
        """Step on streams of the device's greatest (True) or least (False,
        the default) scheduling priority; waits for queued steps first."""
        check(lib().nls_pool_set_priority(self._p, 1 if high else 0))

    def time_passes(self, j0: int, j1: int, reps: int):
        """Mean duration (ms) of one Lanczos pass launch over passes j0..j1
        launched back to back as the step issues them, and the grid points
        one launch covers."""
        ms, pts = ctypes.c_float(), ctypes.c_int64()
        check(lib().nls_pool_time_passes(self._p, j0, j1, reps, ctypes.byref(ms), ctypes.byref(pts)))
        return ms.value, pts.value

    def set_step_kernel(self, one_kernel: bool):
        """2-D FP32 Gautschi pools: run each step as one kernel (True) or as
        the launch sequence (False, the default); see nls_pool_set_step_kernel."""
        check(lib().nls_pool_set_step_kernel(self._p, 1 if one_kernel else 0))

    def set_wait_limit(self, polls: int, stall_stage: int = -1):
        """Bounds of the one-kernel step's device waits (nls_pool_set_wait_limit)."""
        check(lib().nls_pool_set_wait_limit(self._p, int(polls), int(stall_stage)))

    def kernels_per_step(self) -> int:
        v = ctypes.c_int32()
        check(lib().nls_pool_kernels_per_step(self._p, ctypes.byref(v)))
        return v.value

    def close(self):
        if self._p:
            lib().nls_pool_destroy(self._p)
            self._p = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["Spec", "Solver", "Pool", "NlsError", "pinned_empty", "KG_GAUTSCHI", "KG_SV", "SP4_SV",
           "SP4_GAUTSCHI", "NLSE_SS2", "NLSE_SEWI", "FP32", "FP64", "reference_phi4_rm"]
