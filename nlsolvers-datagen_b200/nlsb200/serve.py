"""Serving loop for a stream of trajectory requests of mixed kinds and sizes.

The reference runs one trajectory per process invocation (its launchers call a
driver binary per run, scripts/real_launcher_2d.py:143-170). Here one process
keeps one pool per request class (method, dim, Krylov dimension, precision)
and runs continuous batching:
  - requests arrive over time and are queued per class (first come, first
    served within a class);
  - admission is by device memory: every class draws from one budget of
    device bytes, and a request is admitted when its bytes (its padded grid
    points times its class's bytes per point: fields, Krylov basis, snapshot
    frames) fit in what the running requests leave free and its pool has a
    free slot;
  - all running trajectories of a pool advance together; a trajectory leaves
    when its last snapshot has reached the host and its last step ran, and
    its bytes return to the budget;
  - every pool is driven by its own host thread on its own CUDA streams, so the
    classes step independently and their work overlaps on the GPU; a thread
    keeps one chunk of steps queued ahead: it queues chunk i + 1, waits for
    chunk i (a fence on the pool's stream), then polls, releases and admits,
    so the pool's stream never drains while its host thread works, and a new
    request waits at most two chunks.

Latency of a request = completion time - arrival time (wall clock).
"""
from __future__ import annotations

import math
import os
import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import workloads as W
from .solver import FP32, FP64, KG_GAUTSCHI, KG_SV, NLSE_SEWI, NLSE_SS2, SP4_GAUTSCHI, SP4_SV, Pool, Spec, pinned_empty

NF = 2  # device snapshot frames per trajectory (the engine's double buffer)


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
    out_traj: np.ndarray | None = None  # client-owned output buffers (e.g. page-locked)
    out_vel: np.ndarray | None = None

    @property
    def gp_steps(self) -> int:
        return self.spec.n * (self.spec.nt - 1)


def bytes_per_point(method: int, k: int, precision: int) -> int:
    """Device bytes a pool of this class holds per padded grid point (the
    allocations of nls_pool_create): u_hi, u_lo, m, c, the increment d (real
    methods), the Stormer-Verlet ping-pong buffer, the SEWI history and work
    fields, the Krylov basis (two sequences, one for SS2) and NF FP64
    snapshot frames of (u, v) or complex u."""
    cplx = method in (NLSE_SS2, NLSE_SEWI)
    rsz = 8 if precision == FP64 else 4
    esz = rsz * (2 if cplx else 1)
    b = 2 * esz + 2 * rsz
    if not cplx:
        b += rsz
    if method in (KG_SV, SP4_SV):
        b += esz
    if method == NLSE_SEWI:
        b += 4 * esz
    if method in (KG_GAUTSCHI, SP4_GAUTSCHI, NLSE_SS2, NLSE_SEWI):
        b += esz * (1 if method == NLSE_SS2 else 2) * (k - 1)
    return b + 8 * 2 * NF


def padded_points(spec) -> int:
    """Points a trajectory occupies in its pool: rows padded to 32 elements,
    the region rounded to 256 points."""
    n = ((spec.nx + 31) // 32 * 32) * spec.ny * (spec.nz if spec.dim == 3 else 1)
    return (n + 255) // 256 * 256


@dataclass
class PoolClass:
    method: int
    dim: int
    k: int
    precision: int = FP32
    max_slots: int = 32
    capacity_points: int | None = None  # None: the whole memory budget in this class's points
    high_priority: bool = False  # step on the device's greatest stream priority (a latency class)

    @property
    def bytes_per_point(self) -> int:
        return bytes_per_point(self.method, self.k, self.precision)


@dataclass
class ServeStats:
    completed: int
    wall_s: float
    gp_steps: int
    latencies_s: list = field(default_factory=list)
    peak_bytes: int = 0

    def summary(self) -> dict:
        lat = np.array(self.latencies_s) * 1e3
        return {"completed": self.completed, "wall_s": self.wall_s,
                "gp_steps_per_s": self.gp_steps / self.wall_s if self.wall_s > 0 else 0.0,
                "p50_ms": float(np.percentile(lat, 50)) if lat.size else None,
                "p99_ms": float(np.percentile(lat, 99)) if lat.size else None,
                "mean_ms": float(lat.mean()) if lat.size else None,
                "peak_device_bytes": self.peak_bytes}


class Server:
    """Pools by class name; `run(requests)` serves them in arrival order.

    memory_budget: device bytes shared by all classes' running requests.
    threads: one host thread per pool (False: one thread visits the pools in
    turn, the order deterministic, for tests with stand-in pools)."""

    def __init__(self, classes: dict[str, PoolClass], chunk: int = 20, memory_budget: int = 8 << 30,
                 make_pool=None, threads: bool = True):
        self.classes = classes
        self.chunk = chunk
        self.budget = int(memory_budget)
        self.threads = threads

        def default_pool(pc):
            cap = pc.capacity_points or max(self.budget // pc.bytes_per_point, 1 << 16)
            pool = Pool(pc.method, pc.dim, pc.k, pc.precision, cap, pc.max_slots)
            if pc.high_priority:
                pool.set_priority(True)
            return pool
        make_pool = make_pool or default_pool
        self.pools = {name: make_pool(pc) for name, pc in classes.items()}

    def close(self):
        for p in self.pools.values():
            p.close()

    def request_bytes(self, r: Request) -> int:
        return padded_points(r.spec) * self.classes[r.cls].bytes_per_point

    def run(self, requests: list[Request], clock=time.perf_counter, timeout_s: float = 600.0,
            out_dir: str | None = None) -> ServeStats:
        """Serve `requests`; with out_dir, every request's snapshots are also
        streamed to out_dir/req<rid>_traj.npy (and _vel.npy for KG / phi^4) as
        they reach the host, in the reference drivers' .npy layout."""
        for r in requests:
            if self.request_bytes(r) > self.budget:
                raise ValueError(f"request {r.rid} needs {self.request_bytes(r)} device bytes, more than the "
                                 f"budget of {self.budget}")
        st = _RunState(self, requests, clock, out_dir)
        if self.threads:
            st.run_threaded(timeout_s)
        else:
            st.run_sequential(timeout_s)
        wall = clock() - st.t0
        return ServeStats(completed=len(st.done), wall_s=wall, gp_steps=sum(r.gp_steps for r in st.done),
                          latencies_s=[r.t_done - r.arrival for r in st.done], peak_bytes=st.peak)


class _RunState:
    """Queues, running sets and the device-byte ledger of one Server.run."""

    def __init__(self, srv: Server, requests, clock, out_dir):
        self.srv, self.clock, self.out_dir = srv, clock, out_dir
        self.n = len(requests)
        self.pending = deque(sorted(requests, key=lambda r: r.arrival))
        self.queues = {name: deque() for name in srv.classes}
        self.running = {name: {} for name in srv.classes}  # slot -> request
        self.done = []
        self.used = 0
        self.peak = 0
        self.lock = threading.Lock()
        self.cond = threading.Condition(self.lock)
        self.error = None
        self.fences = {name: None for name in srv.classes}  # the queued chunk's fence per pool
        self.t0 = clock()

    def now(self):
        return self.clock() - self.t0

    def release_arrivals(self):
        now = self.now()
        while self.pending and self.pending[0].arrival <= now:
            r = self.pending.popleft()
            self.queues[r.cls].append(r)

    def admit(self, name):
        """Admit queued requests of class `name` while their bytes fit in the
        budget and the pool takes them (FIFO: the head waits for room)."""
        pool = self.srv.pools[name]
        q = self.queues[name]
        while True:
            with self.lock:
                if not q:
                    return
                r = q[0]
                need = self.srv.request_bytes(r)
                if self.used + need > self.srv.budget:
                    return
                self.used += need  # reserved before the (slow) upload
                self.peak = max(self.peak, self.used)
            out = None
            if self.out_dir:
                base = os.path.join(self.out_dir, f"req{r.rid:05d}")
                out = (base + "_traj.npy", None if r.spec.complex else base + "_vel.npy")
            kw = {}
            if out:
                kw["out_npy"] = out
            if r.out_traj is not None:
                kw["traj"] = r.out_traj
                if r.out_vel is not None:
                    kw["vel"] = r.out_vel
            slot = pool.admit(r.spec, r.u0, r.v0, r.m, r.c, **kw)
            with self.lock:
                if slot is None:  # no free slot or pool capacity: wait for a release
                    self.used -= need
                    return
                q.popleft()
                r.slot, r.t_admit = slot, self.now()
                self.running[name][slot] = r

    def collect(self, name):
        pool = self.srv.pools[name]
        for slot, r in list(self.running[name].items()):
            _, finished = pool.poll(slot)
            if finished:
                info = pool.release(slot)
                with self.cond:
                    r.traj = info.traj
                    r.t_done = self.now()
                    del self.running[name][slot]
                    self.done.append(r)
                    self.used -= self.srv.request_bytes(r)
                    self.cond.notify_all()

    def service(self, name, sync):
        """One round of class `name`: admit, queue a chunk of steps, then (sync:
        wait for the chunk queued in the previous round) poll and release."""
        self.admit(name)
        if not self.running[name]:
            return False
        pool = self.srv.pools[name]
        pool.step(self.srv.chunk)
        if sync:
            t = pool.fence()
            if self.fences[name] is not None:
                pool.fence_wait(self.fences[name])
            self.fences[name] = t
        self.collect(name)
        return True

    def run_sequential(self, timeout_s):
        while len(self.done) < self.n:
            if self.now() > timeout_s:
                raise TimeoutError(f"serving run exceeded {timeout_s} s ({len(self.done)}/{self.n} done)")
            self.release_arrivals()
            busy = False
            for name in self.srv.classes:
                busy |= self.service(name, sync=False)
            if not busy and self.pending:  # idle until the next arrival
                time.sleep(max(0.0, min(self.pending[0].arrival - self.now(), 0.05)))

    def _worker(self, name):
        try:
            while True:
                with self.cond:
                    if self.error is not None or len(self.done) >= self.n:
                        return
                if not self.service(name, sync=True):
                    with self.cond:
                        self.cond.wait(timeout=0.002)
        except BaseException as ex:  # surfaced by the dispatching thread
            with self.cond:
                self.error = ex
                self.cond.notify_all()

    def run_threaded(self, timeout_s):
        workers = [threading.Thread(target=self._worker, args=(name,), daemon=True) for name in self.srv.classes]
        for w in workers:
            w.start()
        try:
            while True:
                with self.cond:
                    self.release_arrivals()
                    self.cond.notify_all()
                    if self.error is not None or len(self.done) >= self.n:
                        break
                    if self.now() > timeout_s:
                        self.error = TimeoutError(f"serving run exceeded {timeout_s} s "
                                                  f"({len(self.done)}/{self.n} done)")
                        break
                    wait = 0.005
                    if self.pending:
                        wait = max(0.0, min(self.pending[0].arrival - self.now(), wait))
                    self.cond.wait(timeout=wait)
        finally:
            with self.cond:
                if self.error is None and len(self.done) < self.n:
                    self.error = RuntimeError("serving run stopped")
                self.cond.notify_all()
            for w in workers:
                w.join(timeout=120)
        if self.error is not None and len(self.done) < self.n:
            raise self.error


@dataclass
class RequestPlan:
    """The drawn parameters of one request of the serving mix (no fields yet)."""
    rid: int
    cls: str
    arrival: float
    n: int
    nt: int
    seed: int
    sigma: float = 0.0

    @property
    def dim(self) -> int:
        return 3 if self.cls == "kg3d" else 2

    @property
    def gp_steps(self) -> int:
        return self.n ** self.dim * (self.nt - 1)

    def padded_points(self) -> int:
        n = ((self.n + 31) // 32 * 32) * self.n * (self.n if self.dim == 3 else 1)
        return (n + 255) // 256 * 256


def mixed_plans(count: int, rate_hz: float, seed: int = 0, steps=(500, 5000), scale: float = 1.0) -> list[RequestPlan]:
    """The random draws of the serving mix, in the order mixed_requests makes
    them: per request the arrival gap, the class, the step count, the field
    seed, the grid edge (and sigma for phi^4)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate_hz)
        kind = ["kg2d", "nlse2d", "kg3d", "phi4_2d"][int(rng.integers(0, 4))]
        nt = int(rng.integers(steps[0], steps[1] + 1)) + 1
        s = int(rng.integers(1 << 30))
        if kind == "kg2d":
            n, sigma = max(16, int(rng.integers(64, 301) * scale)), 0.0
        elif kind == "nlse2d":
            n, sigma = max(16, int(rng.integers(64, 257) * scale)), 0.0
        elif kind == "kg3d":
            n, sigma = max(12, int(rng.integers(64, 161) * scale)), 0.0
        else:
            n = max(16, int(rng.integers(64, 301) * scale))
            sigma = float(rng.uniform(0.05, 0.5))
        out.append(RequestPlan(i, kind, t, n, nt, s, sigma))
    return out


def build_request(pl: RequestPlan, ns: int = 10, pinned: bool = False) -> Request:
    """The request of a plan: its problem and seeded fields (and, pinned, its
    page-locked snapshot buffers)."""
    nt, s, n = pl.nt, pl.seed, pl.n
    if pl.cls == "kg2d":
        spec, u0, v0, m, c = W.kg_case(n, 10.0, T=0.01 * nt, nt=nt, ns=ns, k=10, seed=s, precision=FP32)
    elif pl.cls == "nlse2d":
        spec, u0, v0, m, c = W.nlse_case(n, 10.0, T=1e-3 * nt, nt=nt, ns=ns, k=12, seed=s, precision=FP32)
    elif pl.cls == "kg3d":
        spec, u0, v0, m, c = W.kg_case(n, 10.0, T=0.01 * nt, nt=nt, ns=ns, k=10, seed=s, dim=3, precision=FP32)
    else:
        spec, u0, v0, m, c = W.kg_case(n, 10.0, T=0.01 * nt, nt=nt, ns=ns, k=10, seed=s, method=SP4_SV,
                                       precision=FP32, kinks=True)
        dx = 2 * 10.0 / (n - 1)
        spec.p1, spec.q1, spec.p3, spec.q3 = 0.0, 1.0, 0.0, -1.0
        spec.rm, spec.r0 = 0.0, pl.sigma / math.sqrt(spec.dt * dx ** 2)
        m = np.ones(u0.shape)
    req = Request(pl.rid, pl.cls, pl.arrival, spec, u0, v0, m, None)
    if pinned:
        dt = np.complex128 if spec.complex else np.float64
        req.out_traj = pinned_empty((spec.ns,) + spec.shape, dt)
        if not spec.complex:
            req.out_vel = pinned_empty((spec.ns,) + spec.shape)
    return req


def mixed_requests(count: int, rate_hz: float, seed: int = 0, steps=(500, 5000), scale: float = 1.0,
                   ns: int = 10, pinned: bool = False) -> list[Request]:
    """The serving mix: requests uniform over KG 2-D 64^2-300^2, NLSE 2-D
    64^2-256^2, KG 3-D 64^3-160^3 and phi^4 2-D (u_tt = Lu + u - u^3 + sigma xi,
    sigma ~ U(0.05, 0.5), discrete noise sigma xi / sqrt(dt dx^d) with Philox
    keyed by (seed, step, point)); Poisson arrivals at rate_hz; step counts
    uniform in `steps`. `scale` shrinks the grid edges (for short runs).
    pinned: each request brings page-locked snapshot buffers (a client that
    allocated them ahead), so admission registers no memory."""
    return [build_request(pl, ns, pinned) for pl in mixed_plans(count, rate_hz, seed, steps, scale)]


# ------------------------------------------------------------ several GPUs
# Trajectories never interact, so requests are partitioned across GPUs and
# every GPU runs its own server (one process per GPU, its own pools, streams
# and graphs); nothing crosses NVLink on the hot path.

def plan_bytes(pl: RequestPlan) -> int:
    """Device bytes of a plan's request (padded points x its class's bytes per point)."""
    meth = {"kg2d": KG_GAUTSCHI, "nlse2d": NLSE_SS2, "kg3d": KG_GAUTSCHI, "phi4_2d": SP4_SV}[pl.cls]
    k = {"kg2d": 10, "nlse2d": 12, "kg3d": 10, "phi4_2d": 3}[pl.cls]
    return pl.padded_points() * bytes_per_point(meth, k, FP32)


def partition(plans, ndev: int, key: str = "work") -> list[list]:
    """Greedy placement of requests on ndev GPUs, largest first: each goes to
    the GPU with the least load so far. key "work": load = grid-point-steps
    (balances the GPUs' busy time); "bytes": load = device bytes, the
    bin-packing of n (k-1) s of the memory budget. Within a GPU the requests
    keep their arrival order. Deterministic: every rank computes the same
    placement from the same plans."""
    if ndev < 1:
        raise ValueError("ndev must be at least 1")
    weight = (lambda p: p.gp_steps) if key == "work" else plan_bytes if key == "bytes" else None
    if weight is None:
        raise ValueError(f"unknown placement key {key!r}")
    load = [0] * ndev
    parts = [[] for _ in range(ndev)]
    for pl in sorted(plans, key=lambda p: (-weight(p), p.rid)):
        d = min(range(ndev), key=lambda i: (load[i], i))
        load[d] += weight(pl)
        parts[d].append(pl)
    for part in parts:
        part.sort(key=lambda p: (p.arrival, p.rid))
    return parts


def serve_rank(plans, rank: int, world: int, key: str = "work", ns: int = 10, pinned: bool = False,
               classes=None, **server_kw) -> tuple[list[Request], ServeStats]:
    """The share of GPU `rank` of a stream placed over `world` GPUs: builds only
    its own requests and serves them with a Server on the current device (the
    caller selects it, one process per GPU). Returns the requests (with their
    results) and the rank's stats; the aggregate over ranks is the sum of
    grid-point-steps over the longest wall time."""
    mine = partition(plans, world, key)[rank]
    reqs = [build_request(pl, ns, pinned) for pl in mine]
    if not reqs:
        return [], ServeStats(completed=0, wall_s=0.0, gp_steps=0)
    srv = Server(classes or default_classes(reqs), **server_kw)
    try:
        st = srv.run(reqs)
    finally:
        srv.close()
    return reqs, st


def merge_stats(stats: list[ServeStats]) -> dict:
    """Aggregate of per-GPU stats: completed requests, grid-point-steps over the
    longest wall time, latency percentiles over all requests."""
    lat = [x for st in stats for x in st.latencies_s]
    merged = ServeStats(completed=sum(st.completed for st in stats), wall_s=max(st.wall_s for st in stats),
                        gp_steps=sum(st.gp_steps for st in stats), latencies_s=lat,
                        peak_bytes=max(st.peak_bytes for st in stats))
    out = merged.summary()
    out["per_gpu_gp_steps"] = [st.gp_steps for st in stats]
    out["per_gpu_wall_s"] = [st.wall_s for st in stats]
    return out


def default_classes(requests: list[Request], max_slots: int = 32) -> dict[str, PoolClass]:
    """One pool per class present in `requests` (KG 2-D and 3-D with k = 10,
    NLSE 2-D SS2 with k = 12, phi^4 2-D Stormer-Verlet), up to max_slots
    trajectories each; their points come from the shared memory budget."""
    method = {"kg2d": (KG_GAUTSCHI, 2, 10), "nlse2d": (NLSE_SS2, 2, 12), "kg3d": (KG_GAUTSCHI, 3, 10),
              "phi4_2d": (SP4_SV, 2, 3)}
    out = {}
    for name, (meth, dim, k) in method.items():
        rs = [r for r in requests if r.cls == name]
        if rs:
            out[name] = PoolClass(meth, dim, k, FP32, max_slots=min(max_slots, len(rs)))
    return out
