"""The evaluation of f(T)e_1 that the f(T) kernel uses (ftri_fast in
csrc/nls_kernels.cuh), restated in numpy and checked on CPU against a dense
eigendecomposition of the same tridiagonal matrix, with f applied to |lambda|
for the square-root kinds as the reference does (matfunc_real.hpp:212-238).

    f(T)e_1 = g(T)e_1 + (f - g)(lambda_1) z_1[0] z_1

g is the entire function equal to f on lambda >= 0, summed as a Taylor series
of tridiagonal products; lambda_1 is the truncated Lanczos matrix's negative
eigenvalue (Laguerre's method from the left of the Gershgorin interval, with a
Sturm count that it is the only one below -1e-12 rho) and z_1 comes from the
leading minors at lambda_1. The matrices are the oracle's Lanczos matrices of
Gaussian fields and of their cubes under the no-flux Laplacian, with the
reference's quirks (last diagonal 0), for k = 6..16 and all four kinds.
Bound: 1e-13 relative (measured about 3e-15).
"""
import math

import numpy as np
import pytest

from oracle import oracle as O


def dense_f(d, e, kind, t):
    A = np.diag(d) + np.diag(e, -1) + np.diag(e, 1)
    w, Z = np.linalg.eigh(A)
    if kind == "cos":
        f = np.cos(t * np.sqrt(np.abs(w)))
    elif kind == "sinc2":
        x = t * np.sqrt(np.abs(w))
        f = np.where(np.abs(x) < 1e-8, 1.0, (np.sin(x) / np.where(x == 0, 1, x)) ** 2)
    elif kind == "exp":
        f = np.exp(1j * t * w)
    else:
        v = t * w
        f = np.where(np.abs(v) < 1e-8, 1.0, np.sin(v) / np.where(v == 0, 1, v))
    return Z @ (f * Z[0])


def taylor_f(d, e, kind, t):
    """Returns f(T)e_1, or None where the kernel falls back to QL."""
    k = len(d)
    e_lo = np.concatenate([[0.0], e])
    e_hi = np.concatenate([e, [0.0]])
    rho = np.max(np.abs(d) + e_lo + e_hi)
    sq = kind in ("cos", "sinc2")
    if (t * t * rho if sq else abs(t) * rho) > 4.0:
        return None
    x = np.zeros(k)
    x[0] = 1.0
    c = x.astype(complex)
    a, rpow = 1.0 + 0j, 1.0
    for n in range(1, 81):
        for _ in range(2 if kind == "sinc" else 1):
            x = d * x + e_lo * np.concatenate([[0.0], x[:-1]]) + e_hi * np.concatenate([x[1:], [0.0]])
            rpow *= rho
        if kind == "cos":
            a *= -(t * t) / ((2 * n - 1) * (2 * n))
        elif kind == "sinc2":
            a *= -4 * t * t / ((2 * n + 1) * (2 * n + 2))
        elif kind == "exp":
            a *= 1j * t / n
        else:
            a *= -(t * t) / ((2 * n) * (2 * n + 1))
        c = c + a * x
        if abs(a) * rpow < 1e-18:
            break
    else:
        return None
    if not sq:
        return c

    def minors(xv):
        p = [1.0, d[0] - xv]
        q = [0.0, -1.0]
        r = [0.0, 0.0]
        for i in range(1, k):
            e2, di = e[i - 1] ** 2, d[i] - xv
            p.append(di * p[-1] - e2 * p[-2])
            q.append(di * q[-1] - e2 * q[-2] - p[-2])
            r.append(di * r[-1] - e2 * r[-2] - 2 * q[-2])
        return p, q[-1], r[-1]

    xv = np.min(d - e_lo - e_hi) - 1e-3 * rho - 1e-300
    for _ in range(32):
        p, dp, d2p = minors(xv)
        if p[-1] <= 0:
            break
        G = dp / p[-1]
        H = G * G - d2p / p[-1]
        dx = -k / (G - math.sqrt(max((k - 1) * (k * H - G * G), 0.0)))
        if not dx > 0:
            break
        xv += dx
        if dx <= 2e-16 * abs(xv) + 1e-300:
            break
    else:
        return None
    lam1, dl = xv, 1e-12 * rho
    if lam1 >= -dl:
        return c
    ps, _, _ = minors(-dl)
    if any(v == 0 for v in ps) or sum((ps[i + 1] < 0) != (ps[i] < 0) for i in range(k)) != 1:
        return None
    p1, _, _ = minors(lam1)
    E = np.concatenate([[1.0], np.cumprod(e)])
    u = np.array([(-1) ** i * p1[i] / E[i] for i in range(k)])
    xa = t * math.sqrt(-lam1)
    if kind == "cos":
        corr = math.cos(xa) - math.cosh(xa)
    else:
        corr = (math.sin(xa) / xa) ** 2 - (math.sinh(xa) / xa) ** 2
    return c + corr * u / np.dot(u, u)


KINDS = {"cos": O.F_COS_SQRT, "sinc2": O.F_SINC2_SQRT, "exp": O.F_EXP, "sinc": O.F_SINC}


@pytest.mark.parametrize("kind", list(KINDS))
def test_taylor_f_of_T_matches_dense(kind):
    rng = np.random.default_rng({"cos": 1, "sinc2": 2, "exp": 3, "sinc": 4}[kind])
    worst, used = 0.0, 0
    for trial in range(40):
        n = int(rng.integers(16, 40))
        k = int(rng.integers(6, 17))
        L = float(rng.uniform(5, 15))
        h = 2 * L / (n - 1)
        g = np.linspace(-L, L, n)
        X, Y = np.meshgrid(g, g, indexing="ij")
        u = rng.uniform(0.5, 2) * np.exp(-((X - rng.uniform(-3, 3)) ** 2 + (Y - rng.uniform(-3, 3)) ** 2)
                                        / rng.uniform(0.5, 4))
        if trial % 2:
            u = -u ** 3
        sqk = kind in ("cos", "sinc2")
        t = float(rng.choice([1e-3, 5e-3, 1e-2, 2e-2, 5e-2])) if sqk else float(rng.choice([1e-3, 2e-3, 5e-3]))
        x = u if sqk else u.astype(complex)
        _, T = O.matfunc(x, np.ones_like(u), 2, 1 / h ** 2, -1.0 if sqk else 1.0, k, KINDS[kind],
                         t if kind != "exp" else 1j * t, True)
        T = np.asarray(T)
        d = np.real(np.diag(T)).copy()
        e = np.abs([T[j, j - 1] for j in range(1, k)])
        got = taylor_f(d, e, kind, t)
        if got is None:
            continue
        used += 1
        ref = dense_f(d, e, kind, t)
        worst = max(worst, np.linalg.norm(got - ref) / np.linalg.norm(ref))
    assert used >= 30, used
    assert worst < 1e-13, worst
