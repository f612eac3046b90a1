"""The oracle's restatement of the reference's linear-interpolation
downsampling (scripts/downsampling.py:68-103, :215-257) against the golden
vectors made from the reference's own functions
(tests/golden/make_downsampling_golden.py): equal bitwise."""
import os

import numpy as np
import pytest

from oracle import downsample as D

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "downsampling.npz")


def _cases():
    g = np.load(GOLDEN)
    return [(k[:-3], g[k], g[k[:-3] + "_out"], g[k[:-3] + "_L"]) for k in sorted(g) if k.endswith("_in")]


@pytest.mark.parametrize("name,u,ref,L", _cases(), ids=[c[0] for c in _cases()])
def test_oracle_downsampling_equals_reference(name, u, ref, L):
    out = D.downsample_interpolation(u, ref.shape[1:], L)
    assert out.dtype == ref.dtype and out.shape == ref.shape
    assert np.array_equal(out, ref)


def test_linspace_matches_numpy():
    for L, n in [(10.0, 300), (15.0, 128), (7.3, 33), (1.0, 2)]:
        assert np.array_equal(D.linspace(L, n), np.linspace(-L, L, n))


# ---- spectral crop (downsample_fft / downsample_fft_3d)

FFT_GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "fft_downsampling.npz")


def _fft_cases():
    g = np.load(FFT_GOLDEN)
    return [(k[:-3], g[k], g[k[:-3] + "_out"]) for k in sorted(g) if k.endswith("_in")]


@pytest.mark.parametrize("name,u,ref", _fft_cases(), ids=[c[0] for c in _fft_cases()])
def test_oracle_fft_downsampling_equals_reference(name, u, ref):
    out = D.downsample_fft(u, ref.shape[1:])
    assert out.dtype == ref.dtype and out.shape == ref.shape
    assert np.linalg.norm(out - ref) <= 1e-13 * np.linalg.norm(ref)


def crop_matrix(n, t):
    """The engine's per-axis map (csrc/nls_fft_downsample.cuh, fft_crop_matrix),
    restated: D[q, p] = 1/sqrt(n t) sum_m exp(2 pi i m q / t)
    exp(-2 pi i f(m) p / n), f(m) = (s + ((m + t//2) mod t) - n//2) mod n."""
    s = (n - t) // 2
    m = np.arange(t)
    f = (s + (m + t // 2) % t - n // 2) % n
    H = np.exp(-2j * np.pi * ((f[:, None] * np.arange(n)[None, :]) % n) / n) / np.sqrt(n)
    G = np.exp(2j * np.pi * ((m[None, :] * m[:, None]) % t) / t) / np.sqrt(t)
    return G @ H


@pytest.mark.parametrize("name,u,ref", _fft_cases(), ids=[c[0] for c in _fft_cases()])
def test_crop_matrices_reproduce_reference(name, u, ref):
    """The separable matrix form the device applies, axis by axis, equals the
    reference's FFT pipeline."""
    y = u.astype(np.complex128)
    for ax in range(1, u.ndim):
        D_ = crop_matrix(u.shape[ax], ref.shape[ax])
        y = np.moveaxis(np.tensordot(D_, np.moveaxis(y, ax, 0), axes=(1, 0)), 0, ax)
    if not np.iscomplexobj(u):
        y = y.real
    assert np.linalg.norm(y - ref) <= 1e-12 * np.linalg.norm(ref)
