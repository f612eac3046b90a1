"""Snapshot downsampling on the device (the reference's
scripts/downsampling.py:68-103 and :215-257, which its HDF5 aggregation applies
to every snapshot, scripts/aggregate_single.py:61-76):
  - the drop-in functions (C ABI nls_downsample_linear) against the golden
    vectors made from the reference's own functions: equal bitwise;
  - the fused pool path (nls_pool_set_downsample) against the oracle's
    downsampling of the same run's full-size snapshots: equal bitwise;
and the spectral crop (the reference's downsample_fft / downsample_fft_3d,
scripts/downsampling.py:10-35, :147-178):
  - the drop-ins (C ABI nls_downsample_fft) against the golden vectors made
    from the reference's own functions: within 1e-12 relative (FP64, a direct
    separable transform instead of an FFT, so rounding differs);
  - the fused pool path (nls_pool_set_downsample_fft) against the oracle's
    restatement applied to the same run's full-size snapshots: 1e-12.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "downsampling.npz")


def _cases():
    g = np.load(GOLDEN)
    return [(k[:-3], g[k], g[k[:-3] + "_out"], g[k[:-3] + "_L"]) for k in sorted(g) if k.endswith("_in")]


@pytest.mark.parametrize("name,u,ref,L", _cases(), ids=[c[0] for c in _cases()])
def test_dropin_equals_reference(name, u, ref, L):
    import nlsb200 as nl
    if u.ndim == 3:
        out = nl.downsample_interpolation(u, ref.shape[1:], L[0], L[1])
    else:
        out = nl.downsample_interpolation_3d(u, ref.shape[1:], L[0], L[1], L[2])
    assert out.dtype == ref.dtype and out.shape == ref.shape
    assert np.array_equal(out, ref)


FFT_GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "fft_downsampling.npz")
FFT_TOL = 1e-12


def _fft_cases():
    g = np.load(FFT_GOLDEN)
    return [(k[:-3], g[k], g[k[:-3] + "_out"]) for k in sorted(g) if k.endswith("_in")]


def _rel(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


@pytest.mark.parametrize("name,u,ref", _fft_cases(), ids=[c[0] for c in _fft_cases()])
def test_fft_dropin_against_reference(name, u, ref):
    import nlsb200 as nl
    out = nl.downsample_fft(u, ref.shape[1:]) if u.ndim == 3 else nl.downsample_fft_3d(u, ref.shape[1:])
    assert out.dtype == ref.dtype and out.shape == ref.shape
    assert _rel(out, ref) < FFT_TOL, _rel(out, ref)


def _run(case, target, mode="linear"):
    import nlsb200 as nl
    spec, u0, v0, m, c = case
    cap = ((spec.nx + 31) // 32 * 32) * spec.ny * (spec.nz if spec.dim == 3 else 1) + 256
    out = []
    for ds in (False, True):
        pool = nl.Pool(spec.method, spec.dim, spec.k, spec.precision, capacity_points=cap, max_slots=1)
        s = pool.admit(spec, u0, v0, m, c)
        got = pool.set_downsample(s, target, mode=mode) if ds else None
        while not pool.poll(s)[1]:
            pool.step(10)
        pool.sync()
        info = pool.release(s)
        pool.close()
        out.append(got if ds else (info.traj, info.vel))
    return out


@pytest.mark.parametrize("kind", ["kg2d", "nlse2d", "kg3d"])
def test_fused_snapshot_downsampling(kind):
    import nlsb200 as nl
    from nlsb200 import workloads as W
    from oracle import downsample as D
    if kind == "kg2d":
        case = W.kg_case(48, 10.0, T=0.3, nt=30, ns=3, k=9, seed=3, precision=nl.FP32)
        target = (20, 29)
    elif kind == "nlse2d":
        case = W.nlse_case(40, 8.0, T=0.03, nt=30, ns=3, k=10, seed=4, precision=nl.FP32)
        target = (17, 17)
    else:
        case = W.kg_case(20, 10.0, T=0.2, nt=20, ns=2, k=9, seed=5, dim=3, precision=nl.FP32)
        target = (9, 11, 7)
    spec = case[0]
    (traj, vel), (dtraj, dvel) = _run(case, target)
    L = (spec.Lx, spec.Ly, spec.Lz)[:spec.dim]
    assert np.array_equal(dtraj, D.downsample_interpolation(traj, target, L))
    if vel is not None:
        assert np.array_equal(dvel, D.downsample_interpolation(vel, target, L))


@pytest.mark.parametrize("kind", ["kg2d", "nlse2d", "nlse3d"])
def test_fused_snapshot_fft_downsampling(kind):
    import nlsb200 as nl
    from nlsb200 import workloads as W
    from oracle import downsample as D
    if kind == "kg2d":
        case = W.kg_case(48, 10.0, T=0.3, nt=30, ns=3, k=9, seed=6, precision=nl.FP32)
        target = (20, 29)
    elif kind == "nlse2d":
        case = W.nlse_case(40, 8.0, T=0.03, nt=30, ns=3, k=10, seed=7, precision=nl.FP32)
        target = (17, 16)
    else:  # the 3-D NLSE launcher's choice (scripts/complex_launcher_3d.py:185-187)
        case = W.nlse_case(24, 8.0, T=0.02, nt=20, ns=2, k=10, seed=8, dim=3, precision=nl.FP32)
        target = (12, 9, 10)
    (traj, vel), (dtraj, dvel) = _run(case, target, mode="fft")
    assert _rel(dtraj, D.downsample_fft(traj, target)) < FFT_TOL
    if vel is not None:
        assert _rel(dvel, D.downsample_fft(vel, target)) < FFT_TOL
