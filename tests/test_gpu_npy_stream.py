"""Snapshots streamed to .npy files while later steps run (the output path
after the solver: the reference's drivers write their .npy files only at the
end, kg_driver_dev_2d.cpp:156-158, and its launchers reload them for HDF5).
The files carry the drivers' layout and equal the in-memory results bitwise;
frames appear in them before the run ends."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pool(spec):
    import nlsb200 as nl
    cap = ((spec.nx + 31) // 32 * 32) * spec.ny * (spec.nz if spec.dim == 3 else 1) + 256
    return nl.Pool(spec.method, spec.dim, spec.k, spec.precision, capacity_points=cap, max_slots=1)


@pytest.mark.parametrize("kind", ["kg2d", "nlse2d", "kg2d_downsampled"])
def test_npy_stream_equals_memory(tmp_path, kind):
    import nlsb200 as nl
    from nlsb200 import workloads as W
    if kind.startswith("kg2d"):
        spec, u0, v0, m, c = W.kg_case(40, 10.0, T=0.4, nt=40, ns=8, k=9, seed=11, precision=nl.FP32)
    else:
        spec, u0, v0, m, c = W.nlse_case(36, 8.0, T=0.04, nt=40, ns=8, k=10, seed=12, precision=nl.FP32)
        v0 = None
    # reference run: in memory
    pool = _pool(spec)
    s = pool.admit(spec, u0, v0, m, c)
    if kind.endswith("downsampled"):
        pool.set_downsample(s, (17, 21))
    while not pool.poll(s)[1]:
        pool.step(5)
    info = pool.release(s)
    pool.close()
    mem_t = info.ds_traj if info.ds_traj is not None else info.traj
    mem_v = info.ds_vel if info.ds_traj is not None else info.vel
    # streamed run
    tp, vp = str(tmp_path / "traj.npy"), (None if spec.complex else str(tmp_path / "vel.npy"))
    pool = _pool(spec)
    s = pool.admit(spec, u0, v0, m, c, out_npy=(tp, vp))
    if kind.endswith("downsampled"):
        pool.set_downsample(s, (17, 21))
    seen_partial = False
    while not pool.poll(s)[1]:
        pool.step(5)
        pool.sync()
        ready = pool.stream(s)
        seen_partial |= 1 < ready < spec.ns
    pool.release(s)
    pool.close()
    assert seen_partial  # frames reached the file before the run ended
    ft = np.load(tp)
    assert ft.dtype == mem_t.dtype and ft.shape == mem_t.shape and np.array_equal(ft, mem_t)
    if vp:
        fv = np.load(vp)
        assert fv.shape == mem_v.shape and np.array_equal(fv, mem_v)


def test_serving_loop_writes_request_files(tmp_path):
    from nlsb200 import serve
    reqs = serve.mixed_requests(6, rate_hz=50.0, seed=3, steps=(20, 40), scale=0.25, ns=4)
    srv = serve.Server(serve.default_classes(reqs, max_slots=4), chunk=5)
    try:
        st = srv.run(reqs, out_dir=str(tmp_path))
    finally:
        srv.close()
    assert st.completed == len(reqs)
    for r in reqs:
        f = np.load(os.path.join(str(tmp_path), f"req{r.rid:05d}_traj.npy"))
        assert np.array_equal(f, r.traj)
