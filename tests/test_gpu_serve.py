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


def test_pool_fences():
    """nls_pool_fence / nls_pool_fence_wait: a fence waits for the steps queued
    before it; only the last 16 fences can be waited on; a ticket never issued
    is rejected."""
    import nlsb200 as nl
    from nlsb200 import workloads as W
    sp, u0, v0, m, c = W.kg_case(64, 10.0, T=0.2, nt=20, ns=2, k=10, seed=3, precision=nl.FP32)
    pool = nl.Pool(nl.KG_GAUTSCHI, 2, 10, nl.FP32, capacity_points=1 << 16, max_slots=1)
    slot = pool.admit(sp, u0, v0, m)
    pool.step(5)
    t0 = pool.fence()
    pool.fence_wait(t0)
    assert pool.poll(slot)[0] >= 5
    ts = [pool.fence() for _ in range(16)]
    with pytest.raises(nl.NlsError):
        pool.fence_wait(t0)  # recycled: older than the last 16
    with pytest.raises(nl.NlsError):
        pool.fence_wait(ts[-1] + 1)  # never issued
    pool.fence_wait(ts[0])
    pool.step(20)
    pool.fence_wait(pool.fence())
    pool.sync()
    assert pool.poll(slot)[1]
    pool.release(slot)
    pool.close()


def test_priority_pools_keep_results():
    """nls_pool_set_priority replaces the step's streams between steps (here
    once before the first step and once in the middle of a run); a stream
    served with one high-priority class equals its runs alone bitwise."""
    import nlsb200 as nl
    from nlsb200 import serve
    from nlsb200 import workloads as W
    sp, u0, v0, m, c = W.kg_case(64, 10.0, T=0.3, nt=30, ns=3, k=10, seed=4, precision=nl.FP32)
    res = []
    for switch in (False, True):
        pool = nl.Pool(nl.KG_GAUTSCHI, 2, 10, nl.FP32, capacity_points=1 << 16, max_slots=1)
        if switch:
            pool.set_priority(True)
        slot = pool.admit(sp, u0, v0, m)
        pool.step(12)
        if switch:
            pool.set_priority(False)
        pool.step(40)
        pool.sync()
        assert pool.poll(slot)[1]
        res.append(pool.release(slot).traj)
        pool.close()
    assert np.array_equal(res[0], res[1])
    reqs = serve.mixed_requests(10, rate_hz=300.0, seed=13, steps=(20, 50), scale=0.25, ns=3)
    classes = serve.default_classes(reqs, max_slots=8)
    name = sorted(classes)[0]
    classes[name].high_priority = True
    srv = serve.Server(classes, chunk=6, memory_budget=1 << 30)
    st = srv.run(reqs, timeout_s=300)
    srv.close()
    assert st.completed == len(reqs)
    for r in reqs:
        if r.cls != name:
            continue
        with nl.Solver(r.spec, r.u0, r.v0, r.m, r.c) as sol:
            sol.run()
            traj, _ = sol.snapshots()
        assert np.array_equal(traj, r.traj), r.cls


def test_rank_share_of_a_placed_stream():
    """serve_rank on one GPU: the share of rank 0 of a stream placed over two
    GPUs completes, and its results equal solo runs bitwise (each GPU of a
    multi-GPU server runs the same Server over its own requests)."""
    import nlsb200 as nl
    from nlsb200 import serve
    plans = serve.mixed_plans(12, 200.0, seed=21, steps=(30, 80), scale=0.3)
    share = serve.partition(plans, 2)[0]
    reqs, st = serve.serve_rank(plans, 0, 2, ns=3, chunk=8, memory_budget=1 << 30)
    assert [r.rid for r in reqs] == [p.rid for p in share]
    assert st.completed == len(share) and st.gp_steps == sum(p.gp_steps for p in share)
    for r in reqs[:3]:
        with nl.Solver(r.spec, r.u0, r.v0, r.m, r.c) as sol:
            sol.run()
            traj, _ = sol.snapshots()
        assert np.array_equal(traj, r.traj), r.cls
