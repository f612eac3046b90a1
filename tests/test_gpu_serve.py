"""The serving loop on the GPU: a short mixed stream (KG 2-D, NLSE 2-D, KG 3-D,
phi^4 2-D) through one pool per class. Every request completes, and one request
of each class equals, bitwise, the same trajectory run alone through Solver
(a trajectory's arithmetic does not depend on what shares its pool)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_mixed_stream_completes_and_matches_solo_runs():
    import nlsb200 as nl
    from nlsb200 import serve
    reqs = serve.mixed_requests(12, rate_hz=200.0, seed=11, steps=(30, 80), scale=0.3, ns=4)
    srv = serve.Server(serve.default_classes(reqs, max_slots=8), chunk=8, memory_budget=1 << 30)
    st = srv.run(reqs, timeout_s=300)
    srv.close()
    assert st.completed == len(reqs)
    s = st.summary()
    assert s["p50_ms"] > 0 and s["p99_ms"] >= s["p50_ms"]
    seen = set()
    for r in reqs:
        if r.cls in seen:
            continue
        seen.add(r.cls)
        with nl.Solver(r.spec, r.u0, r.v0, r.m, r.c) as sol:
            sol.run()
            traj, _ = sol.snapshots()
        assert np.array_equal(traj, r.traj), r.cls


def test_memory_budget_bounds_the_running_set():
    """With a device budget of about two requests' bytes the stream still
    completes, the running set never exceeds the budget, and every result
    equals its run alone bitwise."""
    import nlsb200 as nl
    from nlsb200 import serve
    reqs = serve.mixed_requests(8, rate_hz=500.0, seed=12, steps=(20, 40), scale=0.25, ns=3)
    classes = serve.default_classes(reqs, max_slots=8)
    srv = serve.Server(classes, chunk=5, memory_budget=1 << 30)
    need = max(srv.request_bytes(r) for r in reqs)
    srv.close()
    srv = serve.Server(classes, chunk=5, memory_budget=2 * need)
    st = srv.run(reqs, timeout_s=300)
    srv.close()
    assert st.completed == len(reqs) and 0 < st.peak_bytes <= 2 * need
    for r in reqs:
        with nl.Solver(r.spec, r.u0, r.v0, r.m, r.c) as sol:
            sol.run()
            traj, _ = sol.snapshots()
        assert np.array_equal(traj, r.traj), r.cls
