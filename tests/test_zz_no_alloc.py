"""nls_gautschi_step_noalloc: the no-allocation Gautschi step, for callers
that cannot allocate device memory (a code that owns and caps the device
memory pool), against the allocating entry points (nls_create / nls_step /
nls_snapshot) and against the FP64 oracle on the same inputs, over two calls
in a row.

Tolerances (rel-L2 of u after each call):
  FP64 : 1e-9
  FP32 : 1e-5  (each call re-enters through FP64 u, u_past; the handle keeps
                its compensated FP32 state between steps)
The module fixture `device_in_use` runs the allocating engine first, so these
calls always share the process's device context with other allocations and
loaded kernels, whatever order the tests run in; the file is also named to be
collected last.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

TOL64 = 1e-9
TOL32 = 1e-5


def _nl():
    import nlsb200
    return nlsb200


def _case(method, prec, with_c, n=128):
    from nlsb200 import workloads as W
    from nlsb200.solver import FP32, FP64
    # cfg1 geometry (128^2, L = 10, dt = 0.01, k = 10); nt = ns = 3 snapshots steps 1 and 2
    spec, u0, v0, m, c = W.kg_case(n, 10.0, T=0.03, nt=3, ns=3, k=10, seed=7,
                                   precision=FP64 if prec == "fp64" else FP32)
    spec.method = method
    if method == _nl().SP4_GAUTSCHI:
        spec.seed = 1234
    rng = np.random.default_rng(11)
    v0 = 0.2 * rng.standard_normal(u0.shape)
    if with_c:
        c = 1.0 + 0.3 * rng.random(u0.shape)
    return spec, u0, v0, m, c


def _noalloc(spec, u, up, m, c, first_step, nsteps):
    import torch
    nl = _nl()
    p = spec.struct(c is not None)
    stream = torch.cuda.current_stream().cuda_stream
    rc = nl.lib().nls_gautschi_step_noalloc(
        ctypes.byref(p), ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(up.data_ptr()),
        ctypes.c_void_p(m.data_ptr()), ctypes.c_void_p(c.data_ptr() if c is not None else None),
        first_step, nsteps, ctypes.c_void_p(stream))
    nl._lib.check(rc)


@pytest.fixture(scope="module")
def device_in_use():
    """Device work through the allocating engine (a pool of two trajectories
    stepped to the end and released) before any no-alloc call of this
    module."""
    nl = _nl()
    from nlsb200 import workloads as W
    cases = [W.kg_case(48, 10.0, T=0.05, nt=5, ns=5, k=8, seed=90 + i, precision=nl.FP32) for i in range(2)]
    pool = nl.Pool(nl.KG_GAUTSCHI, 2, 8, nl.FP32, capacity_points=2 * 64 * 48 + 4096, max_slots=2)
    slots = [pool.admit(*cs) for cs in cases]
    while not all(pool.poll(s)[1] for s in slots):
        pool.step(5)
    pool.sync()
    for s in slots:
        assert np.all(np.isfinite(pool.release(s).traj))
    pool.close()
    return True


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("variant", ["kg", "kg_c", "phi4"])
def test_noalloc_two_calls_match_handle(prec, variant, device_in_use):
    import torch
    from parity_util import run_oracle
    nl = _nl()
    method = nl.SP4_GAUTSCHI if variant == "phi4" else nl.KG_GAUTSCHI
    spec, u0, v0, m, c = _case(method, prec, variant == "kg_c")
    with nl.Solver(spec, u0, v0, m, c if variant == "kg_c" else None) as s:
        s.run()
        traj, _ = s.snapshots()
    otraj, _ = run_oracle(spec, u0, v0, m, c if variant == "kg_c" else None)
    dev = torch.device("cuda:0")
    u = torch.tensor(u0, dtype=torch.float64, device=dev)
    up = torch.tensor(u0 - spec.dt * v0, dtype=torch.float64, device=dev)  # kg_dev.hpp:55-58
    md = torch.tensor(m, dtype=torch.float64, device=dev)
    cd = torch.tensor(c, dtype=torch.float64, device=dev) if variant == "kg_c" else None
    tol = TOL64 if prec == "fp64" else TOL32
    for call in (1, 2):
        _noalloc(spec, u, up, md, cd, first_step=call, nsteps=1)
        got = u.cpu().numpy()
        assert np.all(np.isfinite(got))
        e = rel_l2(got, traj[call])
        assert e < tol, (call, e)
        e = rel_l2(got, otraj[call])
        assert e < tol, ("oracle", call, e)
        # u_past now holds the state before this step
        prev = traj[call - 1]
        assert rel_l2(up.cpu().numpy(), prev) < tol


@pytest.mark.gpu
def test_noalloc_first_step_zero(device_in_use):
    """A call that starts at step index 0 (the natural first loop index) writes
    no snapshot anywhere and gives the same KG step as index 1 (the index keys
    only the phi^4 noise)."""
    import torch
    nl = _nl()
    spec, u0, v0, m, _ = _case(nl.KG_GAUTSCHI, "fp64", False, n=64)
    dev = torch.device("cuda:0")
    md = torch.tensor(m, dtype=torch.float64, device=dev)
    ua = torch.tensor(u0, dtype=torch.float64, device=dev)
    upa = torch.tensor(u0 - spec.dt * v0, dtype=torch.float64, device=dev)
    ub, upb = ua.clone(), upa.clone()
    _noalloc(spec, ua, upa, md, None, 0, 1)
    _noalloc(spec, ub, upb, md, None, 1, 1)
    torch.cuda.synchronize()
    assert torch.equal(ua, ub) and torch.equal(upa, upb)
    _noalloc(spec, ua, upa, md, None, 1, 1)
    assert np.all(np.isfinite(ua.cpu().numpy()))


@pytest.mark.gpu
def test_noalloc_multi_step_call_matches_single_steps(device_in_use):
    import torch
    nl = _nl()
    spec, u0, v0, m, _ = _case(nl.KG_GAUTSCHI, "fp64", False, n=64)
    dev = torch.device("cuda:0")
    md = torch.tensor(m, dtype=torch.float64, device=dev)
    ua = torch.tensor(u0, dtype=torch.float64, device=dev)
    upa = torch.tensor(u0 - spec.dt * v0, dtype=torch.float64, device=dev)
    ub, upb = ua.clone(), upa.clone()
    _noalloc(spec, ua, upa, md, None, 1, 2)
    _noalloc(spec, ub, upb, md, None, 1, 1)
    _noalloc(spec, ub, upb, md, None, 2, 1)
    assert rel_l2(ua.cpu().numpy(), ub.cpu().numpy()) < 1e-12


def _p(spec):
    return spec.struct(False)


def test_noalloc_rejects_oversized_grid_and_other_methods():
    """Size and method checks happen before any device call (no GPU needed)."""
    nl = _nl()
    from nlsb200.solver import FP32, KG_GAUTSCHI, NLSE_SS2, Spec
    buf = (ctypes.c_double * 4)()
    ptr = ctypes.cast(buf, ctypes.c_void_p)
    big = Spec(KG_GAUTSCHI, 2, nx=4000, ny=4000, T=1.0, nt=10, ns=1, k=10, precision=FP32)
    rc = nl.lib().nls_gautschi_step_noalloc(ctypes.byref(_p(big)), ptr, ptr, ptr, None, 1, 1, None)
    assert rc == -6  # NLS_ERR_CAPACITY
    msg = ctypes.create_string_buffer(512)
    nl.lib().nls_last_error(msg, 512)
    assert b"bytes of scratch" in msg.value and b"33554432" in msg.value
    nlse = Spec(NLSE_SS2, 2, nx=64, ny=64, T=1.0, nt=10, ns=1, k=10, precision=FP32)
    assert nl.lib().nls_gautschi_step_noalloc(ctypes.byref(_p(nlse)), ptr, ptr, ptr, None, 1, 1, None) == -1
    three = Spec(KG_GAUTSCHI, 3, nx=16, ny=16, nz=16, T=1.0, nt=10, ns=1, k=10, precision=FP32)
    assert nl.lib().nls_gautschi_step_noalloc(ctypes.byref(_p(three)), ptr, ptr, ptr, None, 1, 1, None) == -1


def test_noalloc_rejects_step_counter_overflow():
    """first_step + nsteps must stay below INT32_MAX (the device step counter
    is an int); checked before any device call (no GPU needed)."""
    nl = _nl()
    from nlsb200.solver import FP64, KG_GAUTSCHI, Spec
    buf = (ctypes.c_double * 4)()
    ptr = ctypes.cast(buf, ctypes.c_void_p)
    sp = Spec(KG_GAUTSCHI, 2, nx=64, ny=64, T=1.0, nt=10, ns=1, k=10, precision=FP64)
    rc = nl.lib().nls_gautschi_step_noalloc(ctypes.byref(_p(sp)), ptr, ptr, ptr, None, 2**31 - 2, 1, None)
    assert rc == -1
    msg = ctypes.create_string_buffer(512)
    nl.lib().nls_last_error(msg, 512)
    assert b"step counter" in msg.value
    assert nl.lib().nls_gautschi_step_noalloc(ctypes.byref(_p(sp)), ptr, ptr, ptr, None, 0, -1, None) == -1


@pytest.mark.gpu
def test_noalloc_refuses_a_capturing_stream(device_in_use):
    """Inside a CUDA graph capture the call returns NLS_ERR_STATE before it
    enqueues anything (it would copy its status to the host and synchronise),
    so the caller's capture stays valid and replays; outside it runs."""
    import torch
    nl = _nl()
    spec, u0, v0, m, _ = _case(nl.KG_GAUTSCHI, "fp64", False, n=64)
    dev = torch.device("cuda:0")
    md = torch.tensor(m, dtype=torch.float64, device=dev)
    ua = torch.tensor(u0, dtype=torch.float64, device=dev)
    upa = torch.tensor(u0 - spec.dt * v0, dtype=torch.float64, device=dev)
    x = torch.zeros(4, device=dev)
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        x.add_(1)  # warm-up outside the capture
    torch.cuda.current_stream().wait_stream(side)
    err = None
    with torch.cuda.graph(g):
        x.add_(1)
        try:
            _noalloc(spec, ua, upa, md, None, 1, 1)
        except nl.NlsError as ex:
            err = ex
    assert err is not None and err.code == -7, err
    g.replay()
    torch.cuda.synchronize()
    assert torch.all(x == 2)
    u_before = ua.clone()
    _noalloc(spec, ua, upa, md, None, 1, 1)
    torch.cuda.synchronize()
    assert not torch.equal(u_before, ua) and torch.all(torch.isfinite(ua))
