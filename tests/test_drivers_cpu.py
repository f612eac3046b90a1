"""Exit codes of the ten drop-in executables, as the reference's drivers give
them: a wrong argument count prints the usage and returns 1
(kg_driver_dev_2d.cpp:19-33), a u0 array of the wrong shape returns 1
(kg_driver_dev_2d.cpp:61-66, nlse_cubic_driver_2d.cpp:53-59), a bad m / c
array ends with a nonzero status (the reference throws, :79-99). All of these
are decided before any device call, so they run without a GPU; on a machine
without one a well-formed call fails loudly with a nonzero status."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

BIN = os.path.join(ROOT, "nlsolvers-datagen_b200", "bin")
# name: (dim, complex)
EXES = {"kg_gautschi_2d_dev": (2, False), "kg_sv_2d_dev": (2, False), "sp4_sv_2d_dev": (2, False),
        "kg_gautschi_3d_dev": (3, False), "kg_sv_3d_dev": (3, False), "sp4_sv_3d_dev": (3, False),
        "nlse_2d_dev": (2, True), "nlse_sewi_2d_dev": (2, True), "nlse_3d_dev": (3, True),
        "nlse_sewi_3d_dev": (3, True)}


def _argv(tmp, dim, cplx, n=8, u0="u0.npy", m="m.npy"):
    grid = [n] * dim + [4.0] * dim
    if cplx:
        return grid + [tmp / u0, tmp / "traj.npy", 0.1, 10, 2, tmp / m, tmp / "c.npy"]
    return grid + [tmp / u0, tmp / "v0.npy", tmp / "traj.npy", tmp / "vel.npy", 0.1, 10, 2, tmp / m, tmp / "c.npy"]


def _files(tmp, dim, cplx, n=8):
    shape = (n,) * dim
    np.save(tmp / "u0.npy", np.zeros(shape, dtype=np.complex128 if cplx else np.float64))
    np.save(tmp / "u0_bad.npy", np.zeros((n + 1,) * dim, dtype=np.complex128 if cplx else np.float64))
    np.save(tmp / "v0.npy", np.zeros(shape))
    np.save(tmp / "m.npy", np.ones(shape))
    np.save(tmp / "m_bad.npy", np.ones((n, n + 2) + (n,) * (dim - 2)))
    np.save(tmp / "c.npy", np.ones(shape))


def _run(exe, args):
    path = os.path.join(BIN, exe)
    if not os.path.exists(path):
        pytest.skip(f"{path} not built")
    return subprocess.run([path] + [str(a) for a in args], capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("exe", sorted(EXES))
def test_wrong_argc_prints_usage_and_returns_1(exe, tmp_path):
    dim, cplx = EXES[exe]
    args = _argv(tmp_path, dim, cplx)
    for bad in (args[:-1], args + ["extra"], []):
        r = _run(exe, bad)
        assert r.returncode == 1 and "Usage:" in r.stderr, (exe, len(bad), r.returncode, r.stderr)


@pytest.mark.parametrize("exe", sorted(EXES))
def test_u0_shape_mismatch_returns_1(exe, tmp_path):
    dim, cplx = EXES[exe]
    _files(tmp_path, dim, cplx)
    r = _run(exe, _argv(tmp_path, dim, cplx, u0="u0_bad.npy"))
    assert r.returncode == 1 and "dimensions mismatch" in r.stderr, (exe, r.returncode, r.stderr)


@pytest.mark.parametrize("exe", sorted(EXES))
def test_m_shape_mismatch_fails(exe, tmp_path):
    dim, cplx = EXES[exe]
    _files(tmp_path, dim, cplx)
    r = _run(exe, _argv(tmp_path, dim, cplx, m="m_bad.npy"))
    assert r.returncode != 0 and "mismatch" in r.stderr, (exe, r.returncode, r.stderr)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
@pytest.mark.parametrize("exe", ["kg_gautschi_2d_dev", "nlse_sewi_3d_dev"])
def test_without_device_fails_loudly(exe, tmp_path):
    dim, cplx = EXES[exe]
    _files(tmp_path, dim, cplx)
    r = _run(exe, _argv(tmp_path, dim, cplx))
    assert r.returncode != 0 and "no CUDA device" in r.stderr, (r.returncode, r.stderr)
    assert not (tmp_path / "traj.npy").exists()
