"""The serving loop's admission, queueing and latency accounting, on CPU with a
stand-in pool (the GPU run of the same loop is in test_gpu_serve.py)."""
import types

import numpy as np
import pytest


class FakePool:
    """Admits while slots are free; a step advances every running slot."""

    def __init__(self, slots, clock):
        self.free = list(range(slots))[::-1]
        self.run = {}
        self.clock = clock
        self.admitted = []

    def admit(self, spec, u0, v0, m, c=None):
        if not self.free:
            return None
        s = self.free.pop()
        self.run[s] = [spec, 0]
        self.admitted.append(spec.tag)
        return s

    def step(self, n):
        self.clock.t += 0.001 * n
        for v in self.run.values():
            v[1] = min(v[1] + n, v[0].nt - 1)

    def poll(self, slot):
        spec, done = self.run[slot]
        return done, done >= spec.nt - 1

    def release(self, slot):
        spec, _ = self.run.pop(slot)
        self.free.append(slot)
        return types.SimpleNamespace(traj=np.full(1, spec.tag))

    def fence(self):
        self.fences = getattr(self, "fences", 0) + 1
        return self.fences

    def fence_wait(self, ticket):
        assert 0 < ticket <= self.fences

    def close(self):
        pass


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


def _req(rid, cls, arrival, nt, nx=10):
    from nlsb200.serve import Request
    spec = types.SimpleNamespace(nt=nt, n=100, tag=rid, nx=nx, ny=10, nz=1, dim=2, complex=False)
    return Request(rid, cls, arrival, spec, None, None, None)


def test_fifo_admission_latency_and_throughput():
    from nlsb200 import serve
    clock = Clock()
    pools = {}

    def make_pool(pc):
        p = FakePool(pc.max_slots, clock)
        pools[pc.method] = p
        return p

    classes = {"a": serve.PoolClass(method=0, dim=2, k=10, max_slots=2),
               "b": serve.PoolClass(method=1, dim=2, k=10, max_slots=1)}
    srv = serve.Server(classes, chunk=10, make_pool=make_pool, threads=False)
    reqs = [_req(0, "a", 0.0, 101), _req(1, "a", 0.0, 51), _req(2, "a", 0.0, 31),
            _req(3, "b", 0.0, 21), _req(4, "b", 0.0, 21)]
    st = srv.run(reqs, clock=clock)
    assert st.completed == 5
    # class a holds two slots: request 2 waits for request 1 (the shorter) to finish
    assert pools[0].admitted == [0, 1, 2]
    r = {q.rid: q for q in reqs}
    assert r[2].t_admit >= r[1].t_done - 1e-12
    assert r[4].t_admit >= r[3].t_done - 1e-12           # one slot in class b
    assert all(q.traj[0] == q.rid for q in reqs)          # each result went to its request
    s = st.summary()
    assert s["p50_ms"] <= s["p99_ms"] and s["gp_steps_per_s"] > 0
    assert st.gp_steps == sum(100 * (q.spec.nt - 1) for q in reqs)


def test_mixed_requests_shapes_and_phi4_form():
    from nlsb200 import serve
    from nlsb200.solver import SP4_SV
    reqs = serve.mixed_requests(12, rate_hz=10.0, seed=3, steps=(20, 40), scale=0.2)
    assert [q.arrival for q in reqs] == sorted(q.arrival for q in reqs)
    for q in reqs:
        assert 21 <= q.spec.nt <= 41
        if q.cls == "phi4_2d":
            assert q.spec.method == SP4_SV and q.spec.q1 == 1.0 and q.spec.q3 == -1.0
            dx = 20.0 / (q.spec.nx - 1)
            sigma = q.spec.r0 * np.sqrt(q.spec.dt * dx * dx)
            assert 0.05 <= sigma <= 0.5
    classes = serve.default_classes(reqs)
    assert set(classes) == {q.cls for q in reqs}


def test_admission_by_shared_device_memory_budget():
    """Two classes share one budget of two requests' bytes: the class-b
    requests wait, with slots free in their pool, until a class-a request
    finishes and its bytes return to the budget."""
    from nlsb200 import serve
    clock = Clock()

    classes = {"a": serve.PoolClass(method=0, dim=2, k=10, max_slots=4),
               "b": serve.PoolClass(method=0, dim=2, k=10, max_slots=4)}
    # a 10 x 10 grid pads to 32 x 10 = 320 -> 512 points
    per = 512 * serve.bytes_per_point(0, 10, serve.FP32)
    srv = serve.Server(classes, chunk=10, make_pool=lambda pc: FakePool(pc.max_slots, clock), threads=False,
                       memory_budget=2 * per)
    reqs = [_req(0, "a", 0.0, 101), _req(1, "a", 0.0, 51), _req(2, "b", 0.0, 31), _req(3, "b", 0.0, 21)]
    st = srv.run(reqs, clock=clock)
    assert st.completed == 4 and st.peak_bytes == 2 * per
    r = {q.rid: q for q in reqs}
    assert r[0].t_admit == r[1].t_admit == 0.0
    assert r[2].t_admit >= r[1].t_done - 1e-12   # waits for bytes, not for a slot
    assert r[3].t_admit >= min(r[0].t_done, r[2].t_done) - 1e-12


def test_bytes_per_point_follows_the_pool_allocations():
    from nlsb200 import serve
    from nlsb200.solver import FP32, FP64, KG_GAUTSCHI, NLSE_SEWI, NLSE_SS2, SP4_SV
    # KG FP32, k = 9: u_hi, u_lo, m, c, d (20 B) + V 2 x 8 x 4 B + 2 snapshot frames of (u, v) FP64
    assert serve.bytes_per_point(KG_GAUTSCHI, 9, FP32) == 20 + 64 + 32
    # NLSE SS2 complex64, k = 12: 2 x 8 + 2 x 4 + 1 x 11 x 8 + 32
    assert serve.bytes_per_point(NLSE_SS2, 12, FP32) == 24 + 88 + 32
    assert serve.bytes_per_point(NLSE_SEWI, 12, FP32) == 24 + 4 * 8 + 2 * 11 * 8 + 32
    assert serve.bytes_per_point(SP4_SV, 3, FP64) == 16 + 16 + 8 + 8 + 32


def test_oversized_request_is_rejected():
    from nlsb200 import serve
    clock = Clock()
    classes = {"a": serve.PoolClass(method=0, dim=2, k=10, max_slots=1)}
    srv = serve.Server(classes, make_pool=lambda pc: FakePool(1, clock), threads=False, memory_budget=1000)
    with pytest.raises(ValueError):
        srv.run([_req(0, "a", 0.0, 11)], clock=clock)
