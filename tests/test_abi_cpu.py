"""CPU-side checks of the product boundary: the C-ABI library loads and exports
every symbol include/nlsb200.h declares, the drivers keep the reference's argv
contract, and without a GPU the product fails loudly (no CPU fallback)."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HDR = os.path.join(ROOT, "include", "nlsb200.h")


def _declared_symbols():
    txt = open(HDR).read()
    return sorted(set(re.findall(r"\b(nls_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def nl():
    import nlsb200
    if not os.path.exists(nlsb200.LIB_PATH):
        nlsb200.build()
    return nlsb200


def test_header_symbols_exported(nl):
    L = nl.lib()
    syms = _declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(nl.SYMBOLS) <= set(syms)


def test_problem_defaults_match_reference_binaries(nl):
    import ctypes
    from nlsb200 import _lib
    want = {(0, 2): 10, (0, 3): 10, (4, 2): 20, (4, 3): 25, (5, 2): 10, (5, 3): 15, (2, 2): 10}
    for (method, dim), k in want.items():
        p = _lib.Problem()
        assert nl.lib().nls_problem_defaults(ctypes.byref(p), method, dim) == 0
        assert p.k == k
    p = _lib.Problem()
    nl.lib().nls_problem_defaults(ctypes.byref(p), nl.KG_GAUTSCHI, 2)
    assert (p.p1, p.p3) == (0.0, -1.0)  # -m u^3
    nl.lib().nls_problem_defaults(ctypes.byref(p), nl.SP4_SV, 2)
    assert (p.p1, p.p3) == (-1.0, 1.0)  # -m (u - u^3 + s xi)


def test_product_defaults_equal_oracle_restatement(nl):
    """Every method's coefficients and k, as the product resolves them for a
    Spec that sets none (nls_problem_defaults plus the phi^4 noise scale),
    equal the oracle's own restatement of the reference
    (oracle.reference_coefficients), including the NLSE p3 = 1."""
    from oracle import oracle as O
    for method in (nl.KG_GAUTSCHI, nl.KG_SV, nl.SP4_SV, nl.SP4_GAUTSCHI, nl.NLSE_SS2, nl.NLSE_SEWI):
        for dim in (2, 3):
            spec = nl.Spec(method=method, dim=dim, nx=41, ny=41, nz=41 if dim == 3 else 1, Lx=7.0, Ly=7.0,
                           Lz=7.0, T=0.3, nt=60, ns=3)
            p = spec.struct(False)
            want = O.reference_coefficients(method, dim, spec.nx, spec.Lx, spec.dt)
            got = dict(k=p.k, p1=p.p1, q1=p.q1, p3=p.p3, q3=p.q3, r0=p.r0, nonlinearity=p.nonlinearity)
            for key, v in got.items():
                assert v == want[key], (method, dim, key, v, want[key])
            assert p.rm == pytest.approx(want["rm"], rel=1e-15, abs=0), (method, dim)
    p = nl.Spec(method=nl.NLSE_SS2, dim=2, nx=8, ny=8).struct(False)
    assert p.p3 == 1.0  # rho = m |u|^2 (nlse_dev.hpp:27)


def test_phi4_noise_scale(nl):
    spec = nl.Spec(method=nl.SP4_SV, dim=2, nx=101, ny=101, Lx=10, Ly=10, T=1.0, nt=100, ns=10)
    dx = 20 / 100
    assert nl.reference_phi4_rm(spec) == pytest.approx(-0.01 * np.sqrt(2 * dx) / 0.01)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_no_device_fails_loudly(nl):
    spec = nl.Spec(method=nl.KG_GAUTSCHI, dim=2, nx=16, ny=16, k=5)
    u = np.zeros((16, 16))
    with pytest.raises(nl.NlsError) as ei:
        nl.Solver(spec, u, u, u, None)
    assert ei.value.code == -5


def test_invalid_arguments_rejected(nl):
    spec = nl.Spec(method=nl.KG_GAUTSCHI, dim=2, nx=16, ny=16, k=40)  # k > 32
    u = np.zeros((16, 16))
    with pytest.raises(nl.NlsError) as ei:
        nl.Solver(spec, u, u, u, None)
    assert ei.value.code == -1
    spec = nl.Spec(method=nl.KG_GAUTSCHI, dim=2, nx=16, ny=16, nt=5, ns=10)  # nt/ns == 0
    with pytest.raises(nl.NlsError):
        nl.Solver(spec, u, u, u, None)


DRIVERS = {"kg_gautschi_2d_dev": 14, "kg_sv_2d_dev": 14, "sp4_sv_2d_dev": 14,
           "kg_gautschi_3d_dev": 16, "kg_sv_3d_dev": 16, "sp4_sv_3d_dev": 16,
           "nlse_2d_dev": 12, "nlse_sewi_2d_dev": 12, "nlse_3d_dev": 14, "nlse_sewi_3d_dev": 14}


@pytest.mark.parametrize("name,argc", sorted(DRIVERS.items()))
def test_driver_argc_contract(nl, name, argc):
    exe = os.path.join(nl.BIN_DIR, name)
    assert os.access(exe, os.X_OK), exe
    r = subprocess.run([exe, "1", "2"], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr


def test_driver_shape_mismatch(nl, tmp_path):
    exe = os.path.join(nl.BIN_DIR, "kg_gautschi_2d_dev")
    u0 = np.zeros((16, 16))
    bad = np.zeros((15, 16))
    for nm, a in [("u0", u0), ("v0", u0), ("m", bad), ("c", u0)]:
        np.save(tmp_path / f"{nm}.npy", a)
    args = [exe, "16", "16", "5", "5", str(tmp_path / "u0.npy"), str(tmp_path / "v0.npy"),
            str(tmp_path / "t.npy"), str(tmp_path / "v.npy"), "1.0", "10", "2",
            str(tmp_path / "m.npy"), str(tmp_path / "c.npy")]
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode != 0 and "mismatch" in r.stderr
    np.save(tmp_path / "u0.npy", u0.astype(np.float32))  # wrong dtype
    np.save(tmp_path / "m.npy", u0)
    r = subprocess.run(args, capture_output=True, text=True)
    assert r.returncode != 0 and "dtype" in r.stderr


def test_npy_roundtrip_cpp(tmp_path):
    """The drivers' .npy reader/writer against numpy (f8 and c16, 2-D/4-D)."""
    src = os.path.join(ROOT, "nlsolvers-datagen_b200", "csrc")
    prog = tmp_path / "rt.cpp"
    prog.write_text('#include "npy.hpp"\n#include <cstdio>\nint main(int, char**v){\n'
                    ' auto a = npy::load(v[1]);\n'
                    ' npy::save(v[2], a.descr, a.shape, a.data.data(), a.data.size());\n'
                    ' std::printf("%s %zu\\n", a.descr.c_str(), a.shape.size()); return 0; }\n')
    exe = tmp_path / "rt"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", src, str(prog), "-o", str(exe)], check=True)
    rng = np.random.default_rng(0)
    for arr in [rng.standard_normal((7, 5)), rng.standard_normal((3, 4, 5, 6)),
                rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)),
                np.zeros((0, 3)), rng.standard_normal(9)]:
        np.save(tmp_path / "in.npy", arr)
        r = subprocess.run([str(exe), str(tmp_path / "in.npy"), str(tmp_path / "out.npy")],
                           capture_output=True, text=True, check=True)
        back = np.load(tmp_path / "out.npy")
        assert back.dtype == arr.dtype and back.shape == arr.shape
        assert np.array_equal(back, arr)
