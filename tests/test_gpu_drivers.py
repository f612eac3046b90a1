"""The drop-in executables end to end on the GPU: .npy inputs in the layout the
reference's launchers write (scripts/real_launcher_2d.py:143-170,
scripts/complex_launcher_2d.py:141-166), the reference's argv, .npy outputs,
compared with the FP64 oracle on the same inputs.

Tolerances (rel-L2 over all snapshots): default precision (FP64) 1e-9;
NLS_PRECISION=fp32 1e-5 (velocity 1e-4).
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _nl():
    import nlsb200
    return nlsb200


def _run(exe, args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([os.path.join(_nl().BIN_DIR, exe)] + [str(a) for a in args], capture_output=True,
                       text=True, env=e, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]


def _oracle(spec, u0, v0, m, c):
    from parity_util import run_oracle
    return run_oracle(spec, u0, v0, m, c)


@pytest.mark.parametrize("prec", ["default", "fp32"])
def test_kg_gautschi_2d_driver(tmp_path, prec):
    nl = _nl()
    from nlsb200 import workloads as W
    spec, u0, v0, m, c = W.kg_case(40, 8.0, T=1.0, nt=100, ns=5, k=10, seed=21,
                                   precision=nl.FP64 if prec == "default" else nl.FP32)
    rng = np.random.default_rng(5)
    v0 = 0.1 * rng.standard_normal(u0.shape)
    c = 1.0 + 0.3 * rng.random(u0.shape)
    for nm, a in (("u0", u0), ("v0", v0), ("m", m), ("c", c)):
        np.save(tmp_path / f"{nm}.npy", a)
    _run("kg_gautschi_2d_dev",
         [40, 40, 8.0, 8.0, tmp_path / "u0.npy", tmp_path / "v0.npy", tmp_path / "traj.npy",
          tmp_path / "vel.npy", 1.0, 100, 5, tmp_path / "m.npy", tmp_path / "c.npy"],
         {} if prec == "default" else {"NLS_PRECISION": "fp32"})
    traj, vel = np.load(tmp_path / "traj.npy"), np.load(tmp_path / "vel.npy")
    assert traj.shape == vel.shape == (5, 40, 40) and traj.dtype == np.float64
    otraj, ovel = _oracle(spec, u0, v0, m, c)
    tol = 1e-9 if prec == "default" else 1e-5
    assert rel_l2(traj, otraj) < tol
    assert rel_l2(vel, ovel) < (1e-9 if prec == "default" else 1e-4)


def test_kg_gautschi_3d_driver_header_and_values(tmp_path):
    nl = _nl()
    from nlsb200 import workloads as W
    spec, u0, v0, m, c = W.kg_case(14, 6.0, T=0.5, nt=50, ns=4, k=10, seed=22, dim=3, precision=nl.FP64)
    for nm, a in (("u0", u0), ("v0", v0), ("m", m), ("c", c)):
        np.save(tmp_path / f"{nm}.npy", a)
    _run("kg_gautschi_3d_dev",
         [14, 14, 14, 6.0, 6.0, 6.0, tmp_path / "u0.npy", tmp_path / "v0.npy", tmp_path / "traj.npy",
          tmp_path / "vel.npy", 0.5, 50, 4, tmp_path / "m.npy", tmp_path / "c.npy"])
    traj = np.load(tmp_path / "traj.npy")
    # the 4-D header (ns, nz, ny, nx); the reference writes {ns, ny, nx} over the same bytes
    assert traj.shape == (4, 14, 14, 14)
    otraj, _ = _oracle(spec, u0, v0, m, c)
    assert rel_l2(traj, otraj) < 1e-9


def test_nlse_2d_driver(tmp_path):
    nl = _nl()
    from nlsb200 import workloads as W
    spec, u0, _, m, c = W.nlse_case(32, 6.0, T=0.05, nt=50, ns=5, k=20, seed=23, precision=nl.FP64)
    for nm, a in (("u0", u0), ("m", m), ("c", c)):
        np.save(tmp_path / f"{nm}.npy", a)
    _run("nlse_2d_dev", [32, 32, 6.0, 6.0, tmp_path / "u0.npy", tmp_path / "traj.npy", 0.05, 50, 5,
                         tmp_path / "m.npy", tmp_path / "c.npy"])
    traj = np.load(tmp_path / "traj.npy")
    assert traj.shape == (5, 32, 32) and traj.dtype == np.complex128
    otraj, _ = _oracle(spec, u0, None, m, c)
    assert rel_l2(traj, otraj) < 1e-9


def test_sp4_sv_2d_driver_seeded(tmp_path):
    nl = _nl()
    from nlsb200 import workloads as W
    spec, u0, v0, m, c = W.kg_case(36, 8.0, T=0.4, nt=80, ns=4, k=10, seed=24, method=nl.SP4_SV,
                                   precision=nl.FP64, kinks=True)
    spec.seed = 987654321
    for nm, a in (("u0", u0), ("v0", v0), ("m", m), ("c", c)):
        np.save(tmp_path / f"{nm}.npy", a)
    _run("sp4_sv_2d_dev",
         [36, 36, 8.0, 8.0, tmp_path / "u0.npy", tmp_path / "v0.npy", tmp_path / "traj.npy",
          tmp_path / "vel.npy", 0.4, 80, 4, tmp_path / "m.npy", tmp_path / "c.npy"],
         {"NLS_SEED": str(spec.seed)})
    traj = np.load(tmp_path / "traj.npy")
    otraj, _ = _oracle(spec, u0, v0, m, c)
    assert rel_l2(traj, otraj) < 1e-9


@pytest.mark.parametrize("exe,kind", [("kg_gautschi_2d_dev", "sine"), ("nlse_2d_dev", "sat")])
def test_driver_nonlinearity_env(tmp_path, exe, kind):
    """NLS_NONLINEARITY turns an executable into one of the solvers the
    reference's build names without sources (sine-Gordon on the Gautschi KG
    executable, saturable NLSE on the SS2 one), in FP64 against the oracle."""
    nl = _nl()
    from nlsb200 import workloads as W
    if exe.startswith("kg"):
        spec, u0, v0, m, c = W.kg_case(32, 8.0, T=0.5, nt=50, ns=5, k=10, seed=31, precision=nl.FP64)
        spec.nonlinearity = nl.NL_SINE
        arrays = (("u0", u0), ("v0", v0), ("m", m), ("c", c))
        args = [32, 32, 8.0, 8.0, tmp_path / "u0.npy", tmp_path / "v0.npy", tmp_path / "traj.npy",
                tmp_path / "vel.npy", 0.5, 50, 5, tmp_path / "m.npy", tmp_path / "c.npy"]
    else:
        spec, u0, v0, m, c = W.nlse_case(32, 6.0, T=0.05, nt=50, ns=5, k=20, seed=32, precision=nl.FP64)
        spec.nonlinearity = nl.NL_SAT
        arrays = (("u0", u0), ("m", m), ("c", np.ones(u0.shape)))
        args = [32, 32, 6.0, 6.0, tmp_path / "u0.npy", tmp_path / "traj.npy", 0.05, 50, 5, tmp_path / "m.npy",
                tmp_path / "c.npy"]
    for nm, a in arrays:
        np.save(tmp_path / f"{nm}.npy", a)
    _run(exe, args, {"NLS_NONLINEARITY": kind})
    traj = np.load(tmp_path / "traj.npy")
    otraj, _ = _oracle(spec, u0, v0, m, c)
    assert rel_l2(traj, otraj) < 1e-9
