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


# ---- the other six executables: argv order of each family, .npy headers, the
# SEWI snapshot rule (snapshots from step 2 on, nlse_dev.hpp:231), against the
# FP64 oracle and, where it is built, the reference's own device code.

def _save(tmp_path, **arrays):
    for nm, a in arrays.items():
        np.save(tmp_path / f"{nm}.npy", a)


@pytest.mark.parametrize("exe,method_name,dim", [("kg_sv_2d_dev", "KG_SV", 2), ("kg_sv_3d_dev", "KG_SV", 3),
                                                 ("sp4_sv_3d_dev", "SP4_SV", 3)])
def test_real_sv_drivers(tmp_path, exe, method_name, dim):
    nl = _nl()
    from nlsb200 import workloads as W
    n, L = (32, 8.0) if dim == 2 else (14, 6.0)
    spec, u0, v0, m, c = W.kg_case(n, L, T=0.2, nt=40, ns=4, k=10, seed=25, dim=dim,
                                   method=getattr(nl, method_name), precision=nl.FP64)
    v0 = 0.1 * np.random.default_rng(6).standard_normal(u0.shape)
    env = {}
    if method_name == "SP4_SV":
        spec.seed = 424242
        env["NLS_SEED"] = str(spec.seed)
    _save(tmp_path, u0=u0, v0=v0, m=m, c=c)
    grid = [n] * dim + [L] * dim
    _run(exe, grid + [tmp_path / "u0.npy", tmp_path / "v0.npy", tmp_path / "traj.npy", tmp_path / "vel.npy",
                      0.2, 40, 4, tmp_path / "m.npy", tmp_path / "c.npy"], env)
    traj, vel = np.load(tmp_path / "traj.npy"), np.load(tmp_path / "vel.npy")
    assert traj.shape == vel.shape == (4,) + (n,) * dim and traj.dtype == np.float64
    otraj, ovel = _oracle(spec, u0, v0, m, c)
    assert rel_l2(traj, otraj) < 1e-9 and rel_l2(vel, ovel) < 1e-9
    from oracle import ref_kg
    if method_name == "KG_SV" and ref_kg.available():
        rt, rv, _ = ref_kg.run(spec, u0, v0, m, 1)
        assert rel_l2(traj, rt) < 1e-9 and rel_l2(vel, rv) < 1e-9


def _nlse_driver(tmp_path, exe, dim, n, L, T, nt, ns, k, seed, env=None):
    nl = _nl()
    from nlsb200 import workloads as W
    method = nl.NLSE_SEWI if "sewi" in exe else nl.NLSE_SS2
    spec, u0, _, _, c = W.nlse_case(n, L, T=T, nt=nt, ns=ns, k=k, seed=seed, dim=dim, method=method,
                                    precision=nl.FP64)
    m = W.mass_field(u0.shape, np.random.default_rng(seed + 1))
    _save(tmp_path, u0=u0, m=m, c=c)
    grid = [n] * dim + [L] * dim
    _run(exe, grid + [tmp_path / "u0.npy", tmp_path / "traj.npy", T, nt, ns, tmp_path / "m.npy",
                      tmp_path / "c.npy"], env)
    traj = np.load(tmp_path / "traj.npy")
    assert traj.shape == (ns,) + (n,) * dim and traj.dtype == np.complex128
    return spec, u0, m, c, traj


def test_nlse_3d_driver(tmp_path):
    from oracle import ref_nlse
    spec, u0, m, c, traj = _nlse_driver(tmp_path, "nlse_3d_dev", 3, 12, 6.0, 0.05, 20, 4, 25, 26)
    otraj, _ = _oracle(spec, u0, None, m, c)
    assert rel_l2(traj, otraj) < 1e-9
    if ref_nlse.available():
        rt, _ = ref_nlse.run(spec, u0, m, 0)
        assert rel_l2(traj, rt) < 1e-9


@pytest.mark.parametrize("exe,dim,n,L", [("nlse_sewi_2d_dev", 2, 24, 8.0), ("nlse_sewi_3d_dev", 3, 12, 6.0)])
def test_nlse_sewi_drivers_reference_order(tmp_path, exe, dim, n, L):
    """The executables' default operand order is the reference's (variant 0),
    which grows without bound: a few steps are compared. Cadence: step 1 is a
    Strang step that stores a snapshot itself when 1 % freq == 0
    (nlse_dev.hpp:206-209, :195), later steps store when step > 1 and
    step % freq == 0 (:231); nt = 6, ns = 3 (freq 2) stores steps 2 and 4."""
    from oracle import ref_nlse
    spec, u0, m, c, traj = _nlse_driver(tmp_path, exe, dim, n, L, 0.06, 6, 3, 10 if dim == 2 else 15, 27)
    assert spec.k == (10 if dim == 2 else 15)
    otraj, _ = _oracle(spec, u0, None, m, c)
    assert np.all(np.isfinite(traj)) and np.all(traj[1:] != 0)
    assert rel_l2(traj, otraj) < 1e-9
    if ref_nlse.available():
        rt, _ = ref_nlse.run(spec, u0, m, 1)
        assert rel_l2(traj, rt) < 1e-9


@pytest.mark.parametrize("exe,dim,n,L", [("nlse_sewi_2d_dev", 2, 32, 8.0), ("nlse_sewi_3d_dev", 3, 12, 6.0)])
def test_nlse_sewi_drivers_corrected_order(tmp_path, exe, dim, n, L):
    spec, u0, m, c, traj = _nlse_driver(tmp_path, exe, dim, n, L, 0.1, 100, 5, 10 if dim == 2 else 15, 28,
                                        {"NLS_SEWI_VARIANT": "corrected"})
    spec.sewi_variant = 1
    otraj, _ = _oracle(spec, u0, None, m, c)
    assert np.all(np.isfinite(traj)) and rel_l2(traj, otraj) < 1e-9
