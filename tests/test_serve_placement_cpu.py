"""Placement of serving requests on several GPUs (CPU): the greedy partition
assigns every request once, balances the load within one request of the
optimum bound, keeps arrival order within a GPU and is the same on every rank;
two gloo ranks each serve their share through stand-in pools and together
complete the stream exactly once."""
import os
import socket
import types

import numpy as np
import pytest
import torch.multiprocessing as mp

from nlsb200 import serve


def test_partition_assigns_each_request_once_and_balances():
    plans = serve.mixed_plans(40, 10.0, seed=4)
    for ndev in (1, 2, 3, 8):
        parts = serve.partition(plans, ndev)
        rids = sorted(p.rid for part in parts for p in part)
        assert rids == list(range(40))
        loads = [sum(p.gp_steps for p in part) for part in parts]
        biggest = max(p.gp_steps for p in plans)
        # greedy largest-first: no GPU exceeds the least loaded one by more than one request
        assert max(loads) - min(loads) <= biggest
        for part in parts:
            arr = [p.arrival for p in part]
            assert arr == sorted(arr)
        assert parts == serve.partition(plans, ndev)  # deterministic


def test_partition_by_bytes():
    plans = serve.mixed_plans(24, 10.0, seed=6)
    parts = serve.partition(plans, 4, key="bytes")
    loads = [sum(serve.plan_bytes(p) for p in part) for part in parts]
    assert max(loads) - min(loads) <= max(serve.plan_bytes(p) for p in plans)
    with pytest.raises(ValueError):
        serve.partition(plans, 0)
    with pytest.raises(ValueError):
        serve.partition(plans, 2, key="points")


def test_plans_match_the_generated_requests():
    plans = serve.mixed_plans(10, 5.0, seed=8, steps=(30, 60), scale=0.2)
    reqs = serve.mixed_requests(10, 5.0, seed=8, steps=(30, 60), scale=0.2, ns=2)
    for pl, r in zip(plans, reqs):
        assert (pl.rid, pl.cls, pl.arrival) == (r.rid, r.cls, r.arrival)
        assert pl.gp_steps == r.gp_steps
        assert pl.padded_points() == serve.padded_points(r.spec)


def test_merge_stats():
    a = serve.ServeStats(completed=2, wall_s=1.0, gp_steps=100, latencies_s=[0.1, 0.3], peak_bytes=5)
    b = serve.ServeStats(completed=1, wall_s=2.0, gp_steps=300, latencies_s=[0.2], peak_bytes=7)
    m = serve.merge_stats([a, b])
    assert m["completed"] == 3 and m["wall_s"] == 2.0 and m["gp_steps_per_s"] == 200.0
    assert m["per_gpu_gp_steps"] == [100, 300] and m["peak_device_bytes"] == 7


class StepPool:
    """Stand-in pool: every step advances each running slot by one step."""

    def __init__(self, slots):
        self.free = list(range(slots))[::-1]
        self.run = {}

    def admit(self, spec, u0, v0, m, c=None, **kw):
        if not self.free:
            return None
        s = self.free.pop()
        self.run[s] = [spec, 0]
        return s

    def step(self, n):
        for v in self.run.values():
            v[1] = min(v[1] + n, v[0].nt - 1)

    def poll(self, slot):
        spec, done = self.run[slot]
        return done, done >= spec.nt - 1

    def release(self, slot):
        self.run.pop(slot)
        self.free.append(slot)
        return types.SimpleNamespace(traj=np.zeros(1))

    def close(self):
        pass


def _rank(rank, world, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    plans = serve.mixed_plans(14, 200.0, seed=12, steps=(20, 60), scale=0.1)
    reqs, st = serve.serve_rank(plans, rank, world, ns=2, make_pool=lambda pc: StepPool(pc.max_slots),
                                threads=False, chunk=5)
    got = [None] * world
    dist.all_gather_object(got, ([r.rid for r in reqs], st))
    if rank == 0:
        out.put((got, serve.merge_stats([g[1] for g in got])))
    dist.destroy_process_group()


def test_two_ranks_serve_the_stream_once():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, merged = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    rids = sorted(r for ids, _ in got for r in ids)
    assert rids == list(range(14))
    assert all(len(ids) > 0 for ids, _ in got)
    assert merged["completed"] == 14
    plans = serve.mixed_plans(14, 200.0, seed=12, steps=(20, 60), scale=0.1)
    assert merged["per_gpu_gp_steps"] == [sum(p.gp_steps for p in part) for part in serve.partition(plans, 2)]
