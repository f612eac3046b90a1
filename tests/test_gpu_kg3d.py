"""3-D real FP32 Gautschi path (the warp-marching Lanczos passes) against the
FP64 oracle on boxes that exercise its geometry:
  - two x strips (nx > 120 columns), a partial last y band (ny not a multiple
    of the 12 rows of a block), interior and boundary z segments (segment 8);
  - a box narrower than one band and one strip (ny = 5, nx = 7);
  - each trajectory bitwise the same alone and inside a batch.

Tolerance: rel-L2 <= 1e-5 over all snapshots (the FP32 bound), velocity 1e-4.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
TOL32 = 1e-5


def _box_case(nx, ny, nz, seed, nt=20, ns=4, k=10, L=(10.0, 8.0, 9.0), T=0.2):
    import nlsb200 as nl
    from nlsb200 import workloads as W
    rng = np.random.default_rng(seed)
    spec = nl.Spec(method=nl.KG_GAUTSCHI, dim=3, nx=nx, ny=ny, nz=nz, Lx=L[0], Ly=L[1], Lz=L[2], T=T, nt=nt,
                   ns=ns, k=k, precision=nl.FP32, seed=seed)
    z, y, x = np.meshgrid(np.linspace(-L[2], L[2], nz), np.linspace(-L[1], L[1], ny), np.linspace(-L[0], L[0], nx),
                          indexing="ij")
    u0 = np.zeros((nz, ny, nx))
    for _ in range(3):
        a, w = rng.uniform(0.5, 1.5), rng.uniform(1.0, 2.0)
        cz, cy, cx = rng.uniform(-0.5, 0.5, 3) * np.array(L[::-1])
        u0 += a * np.exp(-((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) / (2 * w * w))
    v0 = 0.1 * np.cos(x / L[0]) * np.exp(-(y * y) / 20.0)
    m = W.mass_field(u0.shape, rng)
    return spec, u0, v0, m, None


def _run_pool(cases, segment):
    import nlsb200 as nl
    cap = sum(((s.nx + 31) // 32 * 32) * s.ny * s.nz + 256 for s, *_ in cases)
    pool = nl.Pool(nl.KG_GAUTSCHI, 3, cases[0][0].k, nl.FP32, capacity_points=cap, max_slots=len(cases),
                   segment=segment)
    slots = [pool.admit(*cs) for cs in cases]
    assert None not in slots
    while not all(pool.poll(s)[1] for s in slots):
        pool.step(10)
    pool.sync()
    infos = [pool.release(s) for s in slots]
    pool.close()
    return infos


def _oracle(spec, u0, v0, m, c):
    from parity_util import run_oracle
    return run_oracle(spec, u0, v0, m, c)


@pytest.mark.parametrize("shape,segment", [((130, 29, 41), 8), ((7, 5, 9), 32), ((36, 36, 36), 32)])
def test_kg3d_fp32_boxes(shape, segment):
    case = _box_case(*shape, seed=sum(shape))
    info, = _run_pool([case], segment)
    otraj, ovel = _oracle(*case)
    assert np.all(np.isfinite(info.traj))
    assert rel_l2(info.traj, otraj) < TOL32
    assert rel_l2(info.traj[-1], otraj[-1]) < TOL32
    assert rel_l2(info.vel, ovel) < 1e-4


def test_kg3d_alone_equals_batched():
    cases = [_box_case(*sh, seed=i, nt=12, ns=3) for i, sh in enumerate([(40, 26, 30), (130, 13, 20), (22, 22, 22)])]
    batched = _run_pool(cases, 8)
    for cs, b in zip(cases, batched):
        alone, = _run_pool([cs], 8)
        assert np.array_equal(alone.traj, b.traj) and np.array_equal(alone.vel, b.vel)
