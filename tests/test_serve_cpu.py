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

    def close(self):
        pass


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


def _req(rid, cls, arrival, nt):
    from nlsb200.serve import Request
    spec = types.SimpleNamespace(nt=nt, n=100, tag=rid)
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
    srv = serve.Server(classes, chunk=10, make_pool=make_pool)
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
