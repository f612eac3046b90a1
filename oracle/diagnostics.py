"""FP64 numpy restatement of the reference's post-hoc diagnostics.

TEST INFRASTRUCTURE ONLY: the checker of the device diagnostics
(nls_pool_set_diagnostics); the product never imports it.

Pinned: tests/test_oracle_kat.py checks it against tests/golden/diagnostics.npz,
the outputs of the reference's own functions.
  KG   scripts/compare_utils_real_2d.py:112-131
  NLSE scripts/compare_utils_complex_2d.py:134-151
3-D (no reference function) extends the same central differences to z.
"""
import numpy as np


def _grad_sq(u, h):
    """sum over interior points of sum_axis |central difference|^2 (per point)."""
    inner = tuple(slice(1, -1) for _ in range(u.ndim))
    g = np.zeros(u[inner].shape)
    for ax in range(u.ndim):  # axis 0 is the slowest (z or y), its spacing is h[ax]
        lo = list(inner)
        hi = list(inner)
        lo[ax] = slice(0, -2)
        hi[ax] = slice(2, None)
        d = (u[tuple(hi)] - u[tuple(lo)]) / (2.0 * h[ax])
        g = g + np.abs(d) ** 2
    return g


def spacing(shape, Ls):
    """(h per array axis) with h = 2L/(n-1); shape / Ls in array order."""
    return [2.0 * L / (n - 1) for n, L in zip(shape, Ls)]


def kg(u, v, m, c, Ls):
    """[1/2 sum v^2 dA, 1/2 sum_interior c |grad u|^2 dA, sum m u^4/4 dA, sum u^2 dA]."""
    h = spacing(u.shape, Ls)
    dA = float(np.prod(h))
    inner = tuple(slice(1, -1) for _ in range(u.ndim))
    return np.array([0.5 * np.sum(v ** 2) * dA,
                     0.5 * np.sum(c[inner] * _grad_sq(u, h)) * dA,
                     np.sum(m * (0.25 * u ** 4)) * dA,
                     np.sum(u ** 2) * dA])


def nlse(u, Ls):
    """[sum |u|^2 dA, sum_interior |grad u|^2 dA, -1/2 sum |u|^4 dA, 0]."""
    h = spacing(u.shape, Ls)
    dA = float(np.prod(h))
    return np.array([np.sum(np.abs(u) ** 2) * dA,
                     np.sum(_grad_sq(u, h)) * dA,
                     -0.5 * np.sum(np.abs(u) ** 4) * dA,
                     0.0])
