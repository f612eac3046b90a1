"""The FP64 oracle against dense known answers (numpy / scipy) and the
Random123 Philox4x32-10 known-answer vectors. CPU only.

The reference has no golden vectors (parity unpinned), so these checks pin the
oracle's mathematics: the operator against the CSR assembly of
laplacians.hpp:54-103/158-218, the Lanczos matrix functions against dense
eigendecompositions / expm, the integrators against exact discrete solutions.
"""
import ctypes

import numpy as np
import pytest
import scipy.linalg as sla

from conftest import rel_l2


def dense_operator(shape, c, inv_h2):
    """CSR-equivalent dense matrix of the no-flux FV operator (laplacians.hpp)."""
    n = int(np.prod(shape))
    cf = np.asarray(c, dtype=float).ravel()
    L = np.zeros((n, n))
    strides = []
    s = 1
    for ext in reversed(shape):
        strides.append((s, ext))
        s *= ext
    for i in range(n):
        for st, ext in strides:
            a = (i // st) % ext
            for sg in (-1, 1):
                if 0 <= a + sg < ext:
                    j = i + sg * st
                    cb = (cf[i] + cf[j]) / 2
                    L[i, j] += cb
                    L[i, i] -= cb
    return L * inv_h2


@pytest.mark.parametrize("shape", [(6, 6), (5, 7), (4, 5, 6)])
def test_operator_matches_csr_assembly(oracle_mod, shape):
    rng = np.random.default_rng(1)
    c = 1 + 0.3 * rng.random(shape)
    x = rng.standard_normal(shape)
    L = dense_operator(shape, c, 2.5)
    dim = len(shape)
    y = oracle_mod.apply_operator(x, c, dim, 2.5, -1.0)
    assert np.abs(y.ravel() + L @ x.ravel()).max() < 1e-12
    xc = x + 1j * rng.standard_normal(shape)
    yc = oracle_mod.apply_operator(xc, c, dim, 2.5, 1.0)
    assert np.abs(yc.ravel() - L @ xc.ravel()).max() < 1e-12


def test_tridiag_eig(oracle_mod):
    rng = np.random.default_rng(2)
    for n in (1, 2, 7, 25):
        d = rng.standard_normal(n)
        e = rng.standard_normal(max(n - 1, 0))
        w, Z = oracle_mod.tridiag_eig(d, e)
        T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
        assert np.abs(T @ Z - Z * w).max() < 1e-12
        assert np.abs(Z.T @ Z - np.eye(n)).max() < 1e-12


def test_fT_e1_dense(oracle_mod):
    """f(T) e1 of a symmetric tridiagonal against numpy.linalg.eigh."""
    rng = np.random.default_rng(3)
    k = 10
    d = rng.uniform(1, 50, k)
    e = rng.uniform(0.5, 5, k - 1)
    T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    w, Q = np.linalg.eigh(T)
    for ft, t, f in [(oracle_mod.F_COS_SQRT, 0.1, lambda l, t: np.cos(t * np.sqrt(abs(l)))),
                     (oracle_mod.F_SINC2_SQRT, 0.1, lambda l, t: (np.sin(t * np.sqrt(abs(l))) / (t * np.sqrt(abs(l)))) ** 2),
                     (oracle_mod.F_EXP, 0.05j, lambda l, t: np.exp(t * l)),
                     (oracle_mod.F_SINC, 0.05, lambda l, t: np.sin(t * l) / (t * l))]:
        ref = Q @ (f(w, t) * Q[0, :])
        got = oracle_mod.fT_e1(T, ft, t)
        assert np.abs(got - ref).max() < 1e-13


def test_fT_e1_hermitian_phase(oracle_mod):
    """Complex Hermitian tridiagonal (lower triangle read) equals the dense result."""
    rng = np.random.default_rng(4)
    k = 8
    d = rng.uniform(-5, 5, k)
    s = rng.uniform(0.5, 2, k - 1) * np.exp(1j * rng.uniform(0, 2 * np.pi, k - 1))
    T = np.diag(d).astype(complex) + np.diag(s, -1) + np.diag(np.conj(s), 1)
    w, Q = np.linalg.eigh(T)
    ref = Q @ (np.exp(0.3j * w) * np.conj(Q[0, :]))
    Tl = np.diag(d).astype(complex) + np.diag(s, -1)  # only the lower triangle is read
    got = oracle_mod.fT_e1(Tl, oracle_mod.F_EXP, 0.3j)
    assert np.abs(got - ref).max() < 1e-12


@pytest.mark.parametrize("shape", [(6, 6), (3, 4, 5)])
def test_full_rank_lanczos_is_exact(oracle_mod, shape):
    """k = n with re-orthogonalisation reproduces cos(tau sqrt A) x and exp(i tau L) x."""
    rng = np.random.default_rng(5)
    c = 1 + 0.2 * rng.random(shape)
    x = rng.standard_normal(shape)
    L = dense_operator(shape, c, 3.0)
    n = x.size
    w, Q = np.linalg.eigh(-L)
    tau = 0.07
    ref = Q @ (np.cos(tau * np.sqrt(np.abs(w))) * (Q.T @ x.ravel()))
    y, _ = oracle_mod.matfunc(x, c, len(shape), 3.0, -1.0, n, oracle_mod.F_COS_SQRT, tau)
    assert rel_l2(y.ravel(), ref) < 1e-12
    xc = x + 1j * rng.standard_normal(shape)
    ref = sla.expm(1j * tau * L) @ xc.ravel()
    y, _ = oracle_mod.matfunc(xc, c, len(shape), 3.0, 1.0, 12, oracle_mod.F_EXP, 1j * tau)
    assert rel_l2(y.ravel(), ref) < 1e-10


def test_lanczos_quirks(oracle_mod):
    """T[k-1,k-1] = 0 and the lower subdiagonal holds <A v_j, v_{j-1}>
    (lanczos.hpp:217, 234, 238-239)."""
    rng = np.random.default_rng(6)
    x = rng.standard_normal((8, 8))
    c = np.ones((8, 8))
    k = 6
    _, T = oracle_mod.matfunc(x, c, 2, 1.0, -1.0, k, oracle_mod.F_COS_SQRT, 0.1)
    assert T[k - 1, k - 1] == 0.0
    # the upper subdiagonal carries the norms beta, the lower one the dots
    assert np.all(np.diag(T, 1) > 0)
    assert np.allclose(np.diag(T, -1), np.diag(T, 1), rtol=1e-10)


def test_linear_kg_exact(oracle_mod):
    """m = 0: the Gautschi step is exact for the discrete wave equation
    u'' = L u, so the oracle matches the eigen-decomposed solution."""
    from oracle.oracle import KG_GAUTSCHI, Problem, run
    n, L, T, nt, ns = 8, 3.0, 0.5, 50, 5
    rng = np.random.default_rng(7)
    u0 = rng.standard_normal((n, n))
    v0 = np.zeros((n, n))
    m = np.zeros((n, n))
    c = np.ones((n, n))
    p = Problem(dim=2, nx=n, ny=n, Lx=L, Ly=L, T=T, nt=nt, ns=ns, k=n * n,
                method=KG_GAUTSCHI, p3=-1.0)
    traj, _ = run(p, u0, v0, m, c)
    dx = 2 * L / (n - 1)
    A = -dense_operator((n, n), c, 1 / (dx * dx))
    w, Q = np.linalg.eigh(A)
    dt = T / nt
    freq = nt // ns
    # exact two-step recurrence: u_{n+1} = 2 cos(dt sqrt A) u_n - u_{n-1}, u_{-1} = u0
    cosA = Q @ np.diag(np.cos(dt * np.sqrt(np.abs(w)))) @ Q.T
    u_prev, u = u0.ravel().copy(), u0.ravel().copy()
    for step in range(1, nt):
        u_next = 2 * cosA @ u - u_prev
        # ghost copies (boundaries.cuh): clamp to interior
        g = u_next.reshape(n, n).copy()
        g[0, 1:-1] = g[1, 1:-1]
        g[-1, 1:-1] = g[-2, 1:-1]
        g[:, 0] = g[:, 1]
        g[:, -1] = g[:, -2]
        u_prev, u = u, g.ravel()
        if step % freq == 0 and step // freq < ns:
            assert rel_l2(traj[step // freq].ravel(), u) < 1e-10


def test_philox_random123_kat(oracle_mod):
    L = oracle_mod.lib()
    fn = L.orc_philox4x32_10
    u32 = ctypes.c_uint32
    fn.argtypes = [ctypes.POINTER(u32), ctypes.POINTER(u32), ctypes.POINTER(u32)]
    cases = [
        ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
        ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
        ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
         [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
    ]
    for ctr, key, want in cases:
        c = (u32 * 4)(*ctr)
        k = (u32 * 2)(*key)
        o = (u32 * 4)()
        fn(c, k, o)
        assert list(o) == want


def test_philox_normal_moments(oracle_mod):
    xs = np.array([oracle_mod.philox_normal(11, 3, i) for i in range(20000)])
    assert abs(xs.mean()) < 0.03
    assert abs(xs.std() - 1.0) < 0.03


def test_nlse_ss2_mass_conserved(oracle_mod):
    """SS2 is unitary up to the Krylov error: mass drift is tiny."""
    from oracle.oracle import NLSE_SS2, Problem, run
    n = 24
    rng = np.random.default_rng(8)
    x = np.linspace(-5, 5, n)
    X, Y = np.meshgrid(x, x)
    u0 = np.exp(-(X ** 2 + Y ** 2)) * np.exp(1j * 0.5 * X)
    p = Problem(dim=2, nx=n, ny=n, Lx=5, Ly=5, T=0.5, nt=100, ns=5, k=12, method=NLSE_SS2, p3=1.0)
    traj, _ = run(p, u0, None, np.ones((n, n)), np.ones((n, n)))
    mass = (np.abs(traj) ** 2).sum(axis=(1, 2))
    assert np.abs(mass / mass[0] - 1).max() < 2e-3  # ghost copies change the mass slightly


def test_diagnostics_restatement_matches_reference_functions():
    """The oracle's diagnostics against the golden outputs of the reference's
    own compute_hamiltonian_* / compute_mass* (tests/golden/diagnostics.npz)."""
    import os
    from oracle import diagnostics as D
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "diagnostics.npz"))
    for i in range(2):
        nx, ny, Lx, Ly = g[f"kg{i}_geom"]
        got = D.kg(g[f"kg{i}_u"], g[f"kg{i}_v"], g[f"kg{i}_m"], g[f"kg{i}_c"], (Ly, Lx))
        np.testing.assert_allclose(got, g[f"kg{i}_diag"], rtol=1e-13, atol=0)
        nx, ny, Lx, Ly = g[f"nlse{i}_geom"]
        got = D.nlse(g[f"nlse{i}_u"], (Ly, Lx))
        np.testing.assert_allclose(got, g[f"nlse{i}_diag"], rtol=1e-13, atol=1e-300)


def _reference_bc_copies(u):
    """The reference's ghost copies replayed literally on a flat buffer, in its
    order and with its index convention (device/include/boundaries.cuh:9-19:
    element (i, j) at i*ny + j; :23-81: (x, y, z) at (x*ny + y)*nz + z), for the
    square / cubic grids its drivers accept."""
    f = u.ravel().copy()
    if u.ndim == 2:
        nx = ny = u.shape[0]
        f[0 * ny + 1:0 * ny + 1 + ny - 2] = f[1 * ny + 1:1 * ny + 1 + ny - 2]
        f[(nx - 1) * ny + 1:(nx - 1) * ny + 1 + ny - 2] = f[(nx - 2) * ny + 1:(nx - 2) * ny + 1 + ny - 2]
        for i in range(nx):
            f[i * ny + 0] = f[i * ny + 1]
        for i in range(nx):
            f[i * ny + ny - 1] = f[i * ny + ny - 2]
        return f.reshape(u.shape)
    nx = ny = nz = u.shape[0]
    at = lambda x, y, z: (x * ny + y) * nz + z  # noqa: E731
    for y in range(1, ny - 1):      # x-min / x-max faces, interior y, z
        for z in range(1, nz - 1):
            f[at(0, y, z)] = f[at(1, y, z)]
    for y in range(1, ny - 1):
        for z in range(1, nz - 1):
            f[at(nx - 1, y, z)] = f[at(nx - 2, y, z)]
    for x in range(nx):              # y faces over all x, interior z
        for z in range(1, nz - 1):
            f[at(x, 0, z)] = f[at(x, 1, z)]
    for x in range(nx):
        for z in range(1, nz - 1):
            f[at(x, ny - 1, z)] = f[at(x, ny - 2, z)]
    for x in range(nx):              # z faces over all x, y
        for y in range(ny):
            f[at(x, y, 0)] = f[at(x, y, 1)]
    for x in range(nx):
        for y in range(ny):
            f[at(x, y, nz - 1)] = f[at(x, y, nz - 2)]
    return f.reshape(u.shape)


@pytest.mark.parametrize("shape", [(4, 4), (5, 5), (4, 4, 4), (5, 5, 5)])
def test_ghost_copies_corner_and_edge_order(oracle_mod, shape):
    """Corners and edges come out of the reference's copy order; the oracle
    replays it, and the result is the per-axis clamp to the interior."""
    u = np.arange(1, np.prod(shape) + 1, dtype=np.float64).reshape(shape) * 1.5
    got = oracle_mod.apply_bc(u, len(shape))
    np.testing.assert_array_equal(got, _reference_bc_copies(u))
    idx = np.meshgrid(*[np.clip(np.arange(n), 1, n - 2) for n in shape], indexing="ij")
    np.testing.assert_array_equal(got, u[tuple(idx)])
    uc = u + 1j * u[::-1]
    gotc = oracle_mod.apply_bc(uc, len(shape))
    np.testing.assert_array_equal(gotc, _reference_bc_copies(uc))
