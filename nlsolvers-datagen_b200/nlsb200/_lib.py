"""Loader and ctypes signatures of the C ABI (include/nlsb200.h).

There is no CPU fallback: if lib/libnlsb200.so is missing or cannot be loaded
the import of the solver classes raises.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libnlsb200.so")
BIN_DIR = os.path.join(PKG_ROOT, "bin")

NLS_OK = 0
ERRORS = {
    -1: "invalid argument", -2: "shape mismatch", -3: "out of memory", -4: "CUDA error",
    -5: "no CUDA device", -6: "pool capacity exhausted", -7: "invalid state",
    -8: "numerical failure", -9: "I/O error", -10: "device wait timed out",
}
NLS_ERR_CAPACITY = -6
NLS_ERR_NO_DEVICE = -5

KG_GAUTSCHI, KG_SV, SP4_SV, SP4_GAUTSCHI, NLSE_SS2, NLSE_SEWI = range(6)
# nonlinearity kinds (nls_problem.nonlinearity, include/nlsb200.h)
NL_POLY, NL_SINE, NL_DSINE, NL_SINH, NL_CQ, NL_SAT = range(6)
FP32, FP64 = 0, 1

SYMBOLS = [
    "nls_problem_defaults", "nls_create", "nls_step", "nls_run", "nls_snapshot",
    "nls_steps_done", "nls_destroy", "nls_pool_create", "nls_pool_admit", "nls_pool_step",
    "nls_pool_poll", "nls_pool_release", "nls_pool_sync", "nls_pool_usage",
    "nls_pool_set_graphs", "nls_pool_set_segment", "nls_pool_set_final_segment", "nls_pool_time_pass", "nls_pool_time_passes",
    "nls_pool_kernels_per_step", "nls_pool_destroy", "nls_strerror", "nls_last_error",
    "nls_pool_step_timed", "nls_set_device", "nls_host_alloc", "nls_host_free",
    "nls_gautschi_step_noalloc", "nls_pool_set_diagnostics", "nls_set_diagnostics",
    "nls_pool_set_downsample", "nls_downsample_linear", "nls_pool_snapshots_ready",
    "nls_pool_set_downsample_fft", "nls_downsample_fft", "nls_pool_set_step_kernel", "nls_pool_set_wait_limit",
    "nls_field2d", "nls_pool_fence", "nls_pool_fence_wait", "nls_pool_set_priority",
]


class NlsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, 'error')} ({code}): {msg}")
        self.code = code


class Problem(ctypes.Structure):
    """Mirror of nls_problem."""
    _fields_ = [
        ("dim", ctypes.c_int32), ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
        ("nz", ctypes.c_int32), ("Lx", ctypes.c_double), ("Ly", ctypes.c_double),
        ("Lz", ctypes.c_double), ("T", ctypes.c_double), ("nt", ctypes.c_int32),
        ("ns", ctypes.c_int32), ("k", ctypes.c_int32), ("method", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("sewi_variant", ctypes.c_int32),
        ("has_c", ctypes.c_int32), ("nonlinearity", ctypes.c_int32),
        ("p1", ctypes.c_double), ("q1", ctypes.c_double), ("p3", ctypes.c_double),
        ("q3", ctypes.c_double), ("rm", ctypes.c_double), ("r0", ctypes.c_double),
        ("seed", ctypes.c_uint64),
    ]


def build(quiet: bool = True) -> None:
    """Compile the engine and the drivers with the package Makefile."""
    cmd = ["make", "-C", PKG_ROOT, "-j4"]
    if quiet:
        cmd.insert(1, "-s")
    subprocess.run(cmd, check=True)


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG_ROOT}` "
                           "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    vp, dp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32)
    pp = ctypes.POINTER(Problem)
    i32, i64 = ctypes.c_int32, ctypes.c_int64
    sig = {
        "nls_problem_defaults": [pp, i32, i32],
        "nls_create": [pp, dp, dp, dp, dp, ctypes.POINTER(vp)],
        "nls_step": [vp, i32],
        "nls_run": [vp],
        "nls_snapshot": [vp, dp, dp],
        "nls_steps_done": [vp, ip],
        "nls_destroy": [vp],
        "nls_pool_create": [i32, i32, i32, i32, i64, i32, ctypes.POINTER(vp)],
        "nls_pool_admit": [vp, pp, dp, dp, dp, dp, dp, dp, ip],
        "nls_pool_step": [vp, i32],
        "nls_pool_poll": [vp, i32, ip, ip],
        "nls_pool_release": [vp, i32],
        "nls_pool_sync": [vp],
        "nls_pool_usage": [vp, ip, ctypes.POINTER(i64)],
        "nls_pool_set_graphs": [vp, i32],
        "nls_pool_set_segment": [vp, i32],
        "nls_pool_set_final_segment": [vp, i32],
        "nls_pool_time_pass": [vp, i32, i32, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(i64)],
        "nls_pool_time_passes": [vp, i32, i32, i32, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(i64)],
        "nls_pool_kernels_per_step": [vp, ip],
        "nls_pool_step_timed": [vp, i32, ctypes.POINTER(ctypes.c_float)],
        "nls_pool_destroy": [vp],
        "nls_set_device": [i32],
        "nls_host_alloc": [i64, ctypes.POINTER(vp)],
        "nls_host_free": [vp],
        "nls_last_error": [ctypes.c_char_p, i32],
        "nls_gautschi_step_noalloc": [pp, vp, vp, vp, vp, i32, i32, vp],
        "nls_pool_set_diagnostics": [vp, i32, dp],
        "nls_set_diagnostics": [vp, dp],
        "nls_pool_set_downsample": [vp, i32, ip, dp, dp],
        "nls_downsample_linear": [i32, ctypes.POINTER(i64), ctypes.POINTER(i64), dp, i32, i32, dp, dp],
        "nls_pool_snapshots_ready": [vp, i32, ip],
        "nls_pool_set_downsample_fft": [vp, i32, ip, dp, dp],
        "nls_downsample_fft": [i32, ctypes.POINTER(i64), ctypes.POINTER(i64), i32, i32, dp, dp],
        "nls_pool_set_step_kernel": [vp, i32],
        "nls_pool_set_wait_limit": [vp, i64, i32],
        "nls_field2d": [i32, i32, ctypes.c_double, dp, i32, dp, i32, dp],
        "nls_pool_fence": [vp, ip],
        "nls_pool_fence_wait": [vp, i32],
        "nls_pool_set_priority": [vp, i32],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    L.nls_strerror.argtypes = [ctypes.c_int]
    L.nls_strerror.restype = ctypes.c_char_p
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != NLS_OK:
        buf = ctypes.create_string_buffer(1024)
        lib().nls_last_error(buf, 1024)
        raise NlsError(rc, buf.value.decode(errors="replace"))
