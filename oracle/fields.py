"""CPU restatement (numpy / scipy) of nls_field2d, the device evaluation of the
reference's coefficient fields (scripts/m_fields_2d.py:14-145,
scripts/c_fields_2d.py:12-166), over the same parameter layouts
(include/nlsb200.h, nls_field2d).

TEST INFRASTRUCTURE ONLY: the CPU tests put `evaluate` in place of the device
call to check the product's draws and parameter packing (nlsb200/fields.py)
against tests/golden/fields.npz, the outputs of the reference's own
generators; the GPU tests compare the device with the same fixtures.
"""
import numpy as np
from scipy.ndimage import correlate1d, laplace


def _grid(n, L):
    x = np.linspace(-L, L, n)
    return np.meshgrid(x, x, indexing='ij')


def _gauss(v, P, o):
    taps = int(P[o])
    w = np.asarray(P[o + 1:o + 1 + taps])
    for axis in (0, 1):
        v = correlate1d(v, w, axis, mode='reflect')
    return v, o + 1 + taps


def evaluate(kind, n, L, P, inputs=()):
    P = [float(p) for p in np.asarray(P, dtype=np.float64).ravel()]
    X, Y = _grid(n, L)
    ins = [np.asarray(a, dtype=np.float64).reshape(n, n) for a in inputs]
    if kind == 1:  # m piecewise
        m1, m2, bt, bp, sw = P
        b = [np.sqrt(X ** 2 + Y ** 2) - bp * L, np.maximum(np.abs(X), np.abs(Y)) - bp * L, Y, X, X + Y][int(bt)]
        return m1 + (m2 - m1) * (0.5 * (1 + np.tanh(b / (sw * L))))
    if kind == 2:  # m gradient
        m0, gamma, eps = P
        c = ins[0]
        gx, gy = np.zeros_like(c), np.zeros_like(c)
        gx[1:-1, :] = (c[2:, :] - c[:-2, :]) / 2
        gy[:, 1:-1] = (c[:, 2:] - c[:, :-2]) / 2
        g2 = gx ** 2 + gy ** 2
        return m0 * (1 + gamma * g2 / (g2 + eps ** 2))
    if kind == 3:  # m phase
        m0, delta, sp = P[0], P[1], int(P[2])
        c = ins[0]
        dx = np.roll(c, sp, axis=0) - np.roll(c, -sp, axis=0)
        dy = np.roll(c, sp, axis=1) - np.roll(c, -sp, axis=1)
        mag = np.sqrt(dx ** 2 + dy ** 2)
        return m0 * (1 + delta * (mag / np.max(np.abs(mag))))
    if kind == 4:  # m topological
        m0, eta, lam = P[:3]
        c = ins[0]
        topo = np.sign(laplace(c) - lam * c)
        s, _ = _gauss(topo, P, 3)
        return m0 * (1 + eta * (s / np.max(np.abs(s))))
    if kind == 5:  # m defects
        m0, q = P[0], int(P[1])
        m = np.ones((n, n)) * m0
        for i in range(q):
            x0, y0, st, w = P[2 + 4 * i:6 + 4 * i]
            m += st * np.exp(-((X - x0) ** 2 + (Y - y0) ** 2) / (2 * w ** 2))
        return np.maximum(m, 0.1 * m0)
    if kind in (6, 16):  # quasi-periodic m / c
        base, q = P[0], int(P[1])
        v = np.ones((n, n)) * base
        for i in range(q):
            kx, ky, a, ph = P[2 + 4 * i:6 + 4 * i]
            v += a * np.cos(kx * X + ky * Y + ph)
        if kind == 6:
            return np.maximum(v, 0.1 * base)
        return base * ((v - v.min()) / (v.max() - v.min()))
    if kind == 7:  # m multiscale
        m0, q = P[0], int(P[1])
        m = np.ones((n, n)) * m0
        o = 2
        for i in range(q):
            a = P[o]
            s, o = _gauss(ins[i], P, o + 1)
            m += a * s / np.max(np.abs(s))
        return np.maximum(m, 0.1 * m0)
    if kind == 11:  # c periodic
        base, amp, k = P
        return base * (1 + amp * (np.sin(k * X) * np.sin(k * Y)))
    if kind == 12:  # c piecewise
        nl, base, contrast, lw = int(P[0]), P[1], P[2], P[3]
        v = np.ones((n, n)) * base
        for i in range(nl):
            if i % 2 == 1:
                v[(X >= -L + i * lw) & (X < -L + (i + 1) * lw)] = base * contrast
        return v
    if kind == 13:  # c sign-changing
        base, reg, cs, sh = P
        if int(reg) == 0:
            pat = np.sin(np.pi * X / cs) * np.sin(np.pi * Y / cs)
            return base * np.tanh(sh * pat) if sh > 0 else base * np.sign(pat)
        return base * np.tanh(sh * X / L)
    if kind == 14:  # c layered
        base, q = P[0], int(P[1])
        v = np.ones((n, n)) * base
        for i in range(q):
            cx, cy, a, f, ph = P[2 + 5 * i:7 + 5 * i]
            v += a * np.sin(f * (cx * X + cy * Y) + ph)
        return base * ((v - v.min()) / (v.max() - v.min()))
    if kind == 15:  # c waveguide
        base, ga, q, npts = P[0], P[1], int(P[2]), int(P[3])
        v = np.ones((n, n)) * base
        pts = np.column_stack([X.ravel(), Y.ravel()])
        o = 4
        for i in range(q):
            w = P[o]
            cx, cy = np.asarray(P[o + 1:o + 1 + npts]), np.asarray(P[o + 1 + npts:o + 1 + 2 * npts])
            o += 1 + 2 * npts
            d = np.min(np.sqrt((pts[:, 0:1] - cx[None]) ** 2 + (pts[:, 1:2] - cy[None]) ** 2), axis=1).reshape(n, n)
            v = np.maximum(v, ga * np.exp(-(d ** 2) / (2 * w ** 2)))
        return v
    if kind == 17:  # c turbulent
        base, inten, q = P[0], P[1], int(P[2])
        f = np.zeros((n, n))
        o = 3
        for i in range(q):
            a = P[o]
            s, o = _gauss(ins[i], P, o + 1)
            f += a * s
        f -= np.min(f)
        f /= np.max(f)
        return base * np.exp(inten * (f - 0.5))
    raise ValueError(kind)
