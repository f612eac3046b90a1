"""Serving loop for a stream of trajectory requests of mixed kinds and sizes.

The reference runs one trajectory per process invocation (its launchers call a
driver binary per run, scripts/real_launcher_2d.py:143-170). Here one process
keeps one pool per request class (method, dim, Krylov dimension, precision)
and runs continuous batching. Requests arrive over time and join their class's
pool as soon as it has room (first come, first served within a class). All
running trajectories of a pool advance together. A trajectory leaves its pool
when its last snapshot has reached the host. Every pool has its own CUDA
streams, so stepping several pools back to back overlaps their work on the
GPU.

Latency of a request = completion time - arrival time (wall clock).
"""
from __future__ import annotations

import math
import os
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .solver import FP32, KG_GAUTSCHI, NLSE_SS2, SP4_SV, Pool, Spec
from . import workloads as W


@dataclass
class Request:
    rid: int
    cls: str
    arrival: float          # seconds after the start of the run
    spec: Spec
    u0: np.ndarray
    v0: np.ndarray | None
    m: np.ndarray
    c: np.ndarray | None = None
    t_admit: float = math.nan
    t_done: float = math.nan
    slot: int = -1
    traj: np.ndarray | None = None

    @property
    def gp_steps(self) -> int:
        return self.spec.n * (self.spec.nt - 1)


@dataclass
class PoolClass:
    method: int
    dim: int
    k: int
    precision: int = FP32
    capacity_points: int = 1 << 22
    max_slots: int = 32


@dataclass
class ServeStats:
    completed: int
    wall_s: float
    gp_steps: int
    latencies_s: list = field(default_factory=list)

    def summary(self) -> dict:
        lat = np.array(self.latencies_s) * 1e3
        return {"completed": self.completed, "wall_s": self.wall_s,
                "gp_steps_per_s": self.gp_steps / self.wall_s if self.wall_s > 0 else 0.0,
                "p50_ms": float(np.percentile(lat, 50)) if lat.size else None,
                "p99_ms": float(np.percentile(lat, 99)) if lat.size else None,
                "mean_ms": float(lat.mean()) if lat.size else None}


class Server:
    """Pools by class name; `run(requests)` serves them in arrival order."""

    def __init__(self, classes: dict[str, PoolClass], chunk: int = 10, make_pool=None):
        self.classes = classes
        self.chunk = chunk
        make_pool = make_pool or (lambda pc: Pool(pc.method, pc.dim, pc.k, pc.precision, pc.capacity_points,
                                                  pc.max_slots))
        self.pools = {name: make_pool(pc) for name, pc in classes.items()}

    def close(self):
        for p in self.pools.values():
            p.close()

    def run(self, requests: list[Request], clock=time.perf_counter, timeout_s: float = 600.0,
            out_dir: str | None = None) -> ServeStats:
        """Serve `requests`; with out_dir, every request's snapshots are also
        streamed to out_dir/req<rid>_traj.npy (and _vel.npy for KG / phi^4) as
        they reach the host, in the reference drivers' .npy layout."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        queues = {name: deque() for name in self.classes}
        running = {name: {} for name in self.classes}  # slot -> request
        done = []
        t0 = clock()
        while len(done) < len(requests):
            now = clock() - t0
            if now > timeout_s:
                raise TimeoutError(f"serving run exceeded {timeout_s} s ({len(done)}/{len(requests)} done)")
            while pending and pending[0].arrival <= now:
                r = pending.popleft()
                queues[r.cls].append(r)
            for name, q in queues.items():
                pool = self.pools[name]
                while q:
                    r = q[0]
                    out = None
                    if out_dir:
                        base = os.path.join(out_dir, f"req{r.rid:05d}")
                        out = (base + "_traj.npy", None if r.spec.complex else base + "_vel.npy")
                    slot = pool.admit(r.spec, r.u0, r.v0, r.m, r.c, **({"out_npy": out} if out else {}))
                    if slot is None:
                        break  # full: the request waits for a release
                    q.popleft()
                    r.slot, r.t_admit = slot, clock() - t0
                    running[name][slot] = r
            active = [name for name in self.classes if running[name]]
            if not active:
                if pending:  # idle until the next arrival
                    time.sleep(max(0.0, min(pending[0].arrival - (clock() - t0), 0.05)))
                continue
            for name in active:
                self.pools[name].step(self.chunk)
            for name in active:
                pool = self.pools[name]
                for slot, r in list(running[name].items()):
                    _, finished = pool.poll(slot)
                    if finished:
                        info = pool.release(slot)
                        r.traj = info.traj
                        r.t_done = clock() - t0
                        del running[name][slot]
                        done.append(r)
        wall = clock() - t0
        return ServeStats(completed=len(done), wall_s=wall, gp_steps=sum(r.gp_steps for r in done),
                          latencies_s=[r.t_done - r.arrival for r in done])


def mixed_requests(count: int, rate_hz: float, seed: int = 0, steps=(500, 5000), scale: float = 1.0,
                   ns: int = 10) -> list[Request]:
    """The serving mix: requests uniform over KG 2-D 64^2-300^2, NLSE 2-D
    64^2-256^2, KG 3-D 64^3-160^3 and phi^4 2-D (u_tt = Lu + u - u^3 + sigma xi,
    sigma ~ U(0.05, 0.5), discrete noise sigma xi / sqrt(dt dx^d) with Philox
    keyed by (seed, step, point)); Poisson arrivals at rate_hz; step counts
    uniform in `steps`. `scale` shrinks the grid edges (for short runs)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate_hz)
        kind = ["kg2d", "nlse2d", "kg3d", "phi4_2d"][int(rng.integers(0, 4))]
        nt = int(rng.integers(steps[0], steps[1] + 1)) + 1
        s = int(rng.integers(1 << 30))
        if kind == "kg2d":
            n = max(16, int(rng.integers(64, 301) * scale))
            spec, u0, v0, m, c = W.kg_case(n, 10.0, T=0.01 * nt, nt=nt, ns=ns, k=10, seed=s, precision=FP32)
        elif kind == "nlse2d":
            n = max(16, int(rng.integers(64, 257) * scale))
            spec, u0, v0, m, c = W.nlse_case(n, 10.0, T=1e-3 * nt, nt=nt, ns=ns, k=12, seed=s, precision=FP32)
        elif kind == "kg3d":
            n = max(12, int(rng.integers(64, 161) * scale))
            spec, u0, v0, m, c = W.kg_case(n, 10.0, T=0.01 * nt, nt=nt, ns=ns, k=10, seed=s, dim=3,
                                           precision=FP32)
        else:
            n = max(16, int(rng.integers(64, 301) * scale))
            spec, u0, v0, m, c = W.kg_case(n, 10.0, T=0.01 * nt, nt=nt, ns=ns, k=10, seed=s, method=SP4_SV,
                                           precision=FP32, kinks=True)
            sigma = rng.uniform(0.05, 0.5)
            dx = 2 * 10.0 / (n - 1)
            spec.p1, spec.q1, spec.p3, spec.q3 = 0.0, 1.0, 0.0, -1.0
            spec.rm, spec.r0 = 0.0, sigma / math.sqrt(spec.dt * dx ** 2)
            m = np.ones(u0.shape)
        c = None
        out.append(Request(i, kind, t, spec, u0, v0, m, c))
    return out


def default_classes(requests: list[Request], max_slots: int = 32) -> dict[str, PoolClass]:
    """One pool per class, sized for its largest request x max_slots."""
    method = {"kg2d": (KG_GAUTSCHI, 2, 10), "nlse2d": (NLSE_SS2, 2, 12), "kg3d": (KG_GAUTSCHI, 3, 10),
              "phi4_2d": (SP4_SV, 2, 3)}
    out = {}
    for name, (meth, dim, k) in method.items():
        rs = [r for r in requests if r.cls == name]
        if not rs:
            continue
        big = max(((r.spec.nx + 31) // 32 * 32) * r.spec.ny * (r.spec.nz if dim == 3 else 1) for r in rs)
        slots = min(max_slots, len(rs))
        out[name] = PoolClass(meth, dim, k, FP32, capacity_points=slots * (big + 256), max_slots=slots)
    return out
