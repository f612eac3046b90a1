"""Seeded synthetic inputs with the shapes and distributions of the benchmark
configurations (the reference publishes no dataset; its launchers draw
initial conditions and coefficient fields with numpy, e.g.
scripts/real_launcher_2d.py:78-124).

Grid coordinates follow the drivers: x_i = -L + i dx, dx = 2L/(n-1).

The field generators use numpy only and this module imports nothing else at
load time, so a caller that must not load the engine (the CPU baseline of the
benchmark) can load this file on its own and call kg_fields / nlse_fields; the
*_case helpers add the engine's Spec.
"""
from __future__ import annotations

import numpy as np

# integrator and precision codes (include/nlsb200.h)
KG_GAUTSCHI, NLSE_SS2, FP32 = 0, 4, 0


def axes(dim, n, L):
    x = np.linspace(-L, L, n)
    if dim == 2:
        return np.meshgrid(x, x, indexing="xy")  # (ny, nx), x fastest
    X, Y, Z = np.meshgrid(x, x, x, indexing="xy")
    # meshgrid(xy) gives (ny, nx, nz); reorder to (nz, ny, nx)
    return [np.transpose(a, (2, 0, 1)) for a in (X, Y, Z)]


def grf(shape, rng, power=-3.0):
    """Gaussian random field with power spectrum |k|^power, zero mean, unit std."""
    w = rng.standard_normal(shape)
    ks = np.meshgrid(*[np.fft.fftfreq(s) for s in shape], indexing="ij")
    kk = np.sqrt(sum(k * k for k in ks))
    kk[(0,) * len(shape)] = 1.0
    amp = kk ** (power / 2.0)
    amp[(0,) * len(shape)] = 0.0
    f = np.real(np.fft.ifftn(np.fft.fftn(w) * amp))
    f -= f.mean()
    s = f.std()
    return f / s if s > 0 else f


def mass_field(shape, rng):
    """m(x) = 1 + 0.2 GRF(|k|^-3)."""
    return 1.0 + 0.2 * grf(shape, rng)


def gaussian_bumps(dim, n, L, rng, count=4, amp=(0.5, 2.0), width=(0.5, 2.0), centre=6.0):
    X = axes(dim, n, L)
    u = np.zeros(X[0].shape)
    for _ in range(count):
        a = rng.uniform(*amp)
        w = rng.uniform(*width)
        c = rng.uniform(-centre, centre, size=dim)
        r2 = sum((Xi - ci) ** 2 for Xi, ci in zip(X, c))
        u += a * np.exp(-r2 / (2 * w * w))
    return u


def kink_mix(n, L, rng):
    """Mixture of tanh kink fronts and Gaussian bumps (2-D)."""
    X, Y = axes(2, n, L)
    u = np.zeros(X.shape)
    for _ in range(rng.integers(1, 3)):
        th = rng.uniform(0, 2 * np.pi)
        x0 = rng.uniform(-0.5 * L, 0.5 * L)
        w = rng.uniform(0.5, 2.0)
        u += 0.5 * np.tanh((X * np.cos(th) + Y * np.sin(th) - x0) / w)
    u += gaussian_bumps(2, n, L, rng, count=int(rng.integers(1, 3)), centre=0.6 * L)
    return u


def nlse_solitons(dim, n, L, rng):
    """Sum of 1-3 Gaussian / sech profiles with random phases and velocities."""
    X = axes(dim, n, L)
    u = np.zeros(X[0].shape, dtype=np.complex128)
    for _ in range(rng.integers(1, 4)):
        a = rng.uniform(0.5, 1.5)
        w = rng.uniform(0.8, 2.0)
        c = rng.uniform(-0.5 * L, 0.5 * L, size=dim)
        ph = rng.uniform(0, 2 * np.pi)
        v = rng.uniform(-1, 1, size=dim)
        r = np.sqrt(sum((Xi - ci) ** 2 for Xi, ci in zip(X, c)))
        prof = np.exp(-r * r / (2 * w * w)) if rng.random() < 0.5 else 1.0 / np.cosh(r / w)
        u += a * prof * np.exp(1j * (ph + sum(vi * Xi for vi, Xi in zip(v, X))))
    return u


def kg_fields(n, L, seed=0, dim=2, kinks=False):
    """(u0, v0, m, c) of a KG / phi^4 trajectory with c == 1 (numpy only)."""
    rng = np.random.default_rng(seed)
    u0 = kink_mix(n, L, rng) if kinks else gaussian_bumps(dim, n, L, rng, centre=0.6 * L)
    v0 = np.zeros_like(u0)
    m = mass_field(u0.shape, rng)
    c = np.ones_like(u0)
    return u0, v0, m, c


def nlse_fields(n, L, seed=0, dim=2):
    """(u0, m, c) of an NLSE trajectory with m == c == 1 (numpy only)."""
    rng = np.random.default_rng(seed)
    u0 = nlse_solitons(dim, n, L, rng)
    return u0, np.ones(u0.shape), np.ones(u0.shape)


def kg_case(n, L, T, nt, ns, k=10, seed=0, dim=2, method=KG_GAUTSCHI, precision=FP32,
            kinks=False):
    """(spec, u0, v0, m, c) for a KG / phi^4 trajectory with c == 1."""
    from .solver import Spec
    spec = Spec(method=method, dim=dim, nx=n, ny=n, nz=n if dim == 3 else 1, Lx=L, Ly=L, Lz=L,
                T=T, nt=nt, ns=ns, k=k, precision=precision, seed=seed)
    u0, v0, m, c = kg_fields(n, L, seed, dim, kinks)
    return spec, u0, v0, m, c


def nlse_case(n, L, T, nt, ns, k=12, seed=0, dim=2, method=NLSE_SS2, precision=FP32):
    from .solver import Spec
    spec = Spec(method=method, dim=dim, nx=n, ny=n, nz=n if dim == 3 else 1, Lx=L, Ly=L, Lz=L,
                T=T, nt=nt, ns=ns, k=k, precision=precision, seed=seed)
    u0, m, c = nlse_fields(n, L, seed, dim)
    return spec, u0, None, m, c


# Benchmark configurations (sizes as the reference's headline configs).
CONFIGS = {
    # plain FP64 single trajectory: KG 2-D 128^2 on [-10,10]^2, k=10, dt=0.01, 1000 steps, 10 snapshots
    "kg2d_128_fp64": dict(n=128, L=10.0, T=10.0, nt=1000, ns=10, k=10),
    # batched KG 2-D: 64 x 300^2 on [-15,15]^2, dt=0.005, 6000 steps, 50 snapshots
    "kg2d_300_b64": dict(n=300, L=15.0, T=30.0, nt=6000, ns=50, k=10, batch=64),
    # batched NLSE 2-D: 128 x 200^2 on [-10,10]^2, dt=1e-3, 2000 steps, 100 snapshots, k=12
    "nlse2d_200_b128": dict(n=200, L=10.0, T=2.0, nt=2000, ns=100, k=12, batch=128),
    # batched KG 3-D: 40 x 220^3 on [-10,10]^3, dt=0.01, 10000 steps, 40 snapshots
    "kg3d_220_b40": dict(n=220, L=10.0, T=100.0, nt=10000, ns=40, k=10, batch=40),
}
