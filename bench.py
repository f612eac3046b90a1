#!/usr/bin/env python
"""Benchmark of the batched Lanczos exponential integrator (one JSON line).

Workload (the headline batched configuration): 64 nonlinear Klein-Gordon
trajectories u_tt = Lap u - m u^3 on [-15,15]^2, 300 x 300 grid (incl. ghost
ring), Gautschi step with a k-step Lanczos cos / sinc^2 filter, dt = 0.005,
nt = 6000, 50 snapshots, FP32 Krylov basis + compensated FP32 fields. k = 9:
the project autotuner's choice for this workload (the smallest k in 8..16
whose 10-step result stays within 5e-6 of k = 24), re-checked live and
reported under "tuning". A "step" is one time step of the whole batch.
Inputs are seeded synthetic fields (kink/Gaussian mixtures, m = 1 + 0.2 GRF).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1: one process per GPU (started here through torch.distributed.run when
WORLD_SIZE is unset); every rank steps its own 64 trajectories (weak scaling,
no data-path collective); the step time is the max over ranks.
The timed region is repeated in blocks of exactly K steps until it lasts about
a second (clock samples); the line reports the median block.
--impl reference times the reference algorithm's CPU restatement (the FP64
oracle; the reference itself has no CPU path) on the host cores, rank 0 only,
with the same k and configuration, and reports beside it the reference's own
per-trajectory FP64 GPU path, compiled from its sources, on one trajectory of
the same grid. That arm imports nothing of the engine.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "nlsolvers-datagen_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "grid-point-steps/s batched FP32 vs plain FP64 @rel-L2≤1e-5; HBM GB/s; p50/p99"
UNIT = "grid-point-steps/s"
CFG = dict(n=300, L=15.0, T=30.0, nt=6000, ns=50, batch=64)
K_HEADLINE = 9
FALLBACK_HBM = 6650.0
# DRAM bytes (read + write) per grid point of one Lanczos pass launch
# (k2_lanczos1_f32c, j = 2, both sequences) in the ncu capture of
# profiles/ncu_lanczos_pass_kg2d.md; algorithmic: 24 B per point.
TRAFFIC_BYTES_PER_POINT_PASS = 17.79
TIMED_REGION_S = 1.0
FINAL_ROWS = 25  # rows per tile of the 2-D final pass


def workload_config(k, ws, B):
    """The configuration both arms report (identical keys and values)."""
    return {"workload": "KG 2-D Gautschi batch, 64 x 300^2 on [-15,15]^2, dt=0.005, nt=6000, ns=50",
            "global_batch": B * ws, "per_gpu_batch": B, "grid": [CFG["n"], CFG["n"]], "k": k,
            "parallelism": f"trajectory shards x{ws}",
            "l2": "working set 0.6 GB per GPU >> 126 MB L2 (no flush needed)"}


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


def step_bytes_per_gp(k, s=4, s_m=4, s_c=0):
    """Algorithmic bytes per grid-point-step of the Gautschi step (two Krylov
    sequences sharing passes): every Krylov vector written once, read as the
    stencil input, read as v_{j-1} and read once in the final combination."""
    return s * (8 * k - 8) + 2 * s_m + s_c * (k - 1)


def pass_bytes_per_gp(s=4):
    """Lanczos pass j >= 2 of the Gautschi step: per sequence read V_{j-1} and
    V_{j-2}, write V_j; two sequences."""
    return 2 * 3 * s


class Clocks:
    """SM clock, power and clock-event reasons of this rank's GPU, read through
    NVML (read-only queries) every 2 ms while the timed region runs. The GPU is
    found by the CUDA device's PCI bus id, so the sample is of the device the
    kernels run on whatever CUDA_VISIBLE_DEVICES maps."""

    def __init__(self, index):
        self.index = index
        self.rows = []  # (sm_mhz, max_mhz, reasons bitmask)
        self._stop = threading.Event()
        self._t = None
        self._h = None
        self.device = None

    def _handle(self):
        import pynvml as N
        N.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            self.device = bus
            return N.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            ids = [x for x in vis.split(",") if x.strip().isdigit()]
            idx = int(ids[self.index]) if self.index < len(ids) else self.index
            self.device = f"nvml index {idx}"
            return N.nvmlDeviceGetHandleByIndex(idx)

    def _sample(self):
        import pynvml as N
        sm = N.nvmlDeviceGetClockInfo(self._h, N.NVML_CLOCK_SM)
        mx = N.nvmlDeviceGetMaxClockInfo(self._h, N.NVML_CLOCK_SM)
        rs = N.nvmlDeviceGetCurrentClocksEventReasons(self._h)
        self.rows.append((sm, mx, rs))

    def _run(self):
        while not self._stop.is_set():
            try:
                self._sample()
            except Exception:
                pass
            self._stop.wait(0.002)

    def __enter__(self):
        try:
            self._h = self._handle()
            self._sample()
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        except Exception:
            self._h = None
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if self._h is not None:
            try:
                self._sample()
            except Exception:
                pass

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        import pynvml as N
        names = {N.nvmlClocksEventReasonHwSlowdown: "hw_slowdown",
                 N.nvmlClocksEventReasonHwThermalSlowdown: "hw_thermal_slowdown",
                 N.nvmlClocksEventReasonSwThermalSlowdown: "sw_thermal_slowdown",
                 N.nvmlClocksEventReasonSwPowerCap: "sw_power_cap",
                 N.nvmlClocksEventReasonHwPowerBrakeSlowdown: "hw_power_brake_slowdown"}
        reasons = sorted({nm for _, _, rs in self.rows for bit, nm in names.items() if rs & bit})
        return {"sm_mhz": statistics.median(r[0] for r in self.rows),
                "sm_max_mhz": max(r[1] for r in self.rows), "reasons": reasons,
                "samples": len(self.rows), "source": f"NVML every 2 ms ({self.device})"}


_FIELDS = None


def fields_module():
    """nlsb200/workloads.py loaded on its own (numpy only, no engine import),
    so that the reference arm builds the same inputs without the engine."""
    global _FIELDS
    if _FIELDS is None:
        path = os.path.join(PKG, "nlsb200", "workloads.py")
        spec = importlib.util.spec_from_file_location("nls_bench_fields", path)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _FIELDS = mod
    return _FIELDS


def batch_fields(B, rank):
    """(seed, u0, v0, m, c) of the batch's trajectories on `rank`: seed
    1000 rank + i, kink mixtures for even i."""
    F = fields_module()
    out = []
    for i in range(B):
        seed = 1000 * rank + i
        out.append((seed,) + F.kg_fields(CFG["n"], CFG["L"], seed=seed, kinks=(i % 2 == 0)))
    return out


def make_batch(B, rank, k, nt=None, ns=None, T=None):
    """The batch as engine problems: (Spec, u0, v0, m, c) per trajectory."""
    from nlsb200.solver import FP32, KG_GAUTSCHI, Spec
    cases = []
    for seed, u0, v0, m, c in batch_fields(B, rank):
        spec = Spec(method=KG_GAUTSCHI, dim=2, nx=CFG["n"], ny=CFG["n"], Lx=CFG["L"], Ly=CFG["L"], Lz=CFG["L"],
                    T=T or CFG["T"], nt=nt or CFG["nt"], ns=ns or CFG["ns"], k=k, precision=FP32, seed=seed)
        cases.append((spec, u0, v0, m, c))
    return cases


def oracle_problem(k, seed=0, nt=None, ns=None, T=None):
    """The FP64 oracle's problem for one trajectory of the workload, with the
    reference's KG coefficients (oracle.reference_coefficients); no engine
    import."""
    from oracle import oracle as O
    nt, ns, T = nt or CFG["nt"], ns or CFG["ns"], T or CFG["T"]
    prm = O.reference_coefficients(O.KG_GAUTSCHI, 2, CFG["n"], CFG["L"], T / nt)
    return O.Problem(dim=2, nx=CFG["n"], ny=CFG["n"], nz=1, Lx=CFG["L"], Ly=CFG["L"], Lz=CFG["L"], T=T, nt=nt,
                     ns=ns, k=k, method=O.KG_GAUTSCHI, sewi_variant=0, reorth=1, max_steps=0, p1=prm["p1"],
                     q1=prm["q1"], p3=prm["p3"], q3=prm["q3"], rm=prm["rm"], r0=prm["r0"], seed=seed,
                     nonlinearity=0)


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    lrank = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist
        # host-side plumbing only (barrier, k / segment broadcast, max over
        # ranks of the device timings): the data path has no collective
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    return ws, rank, lrank


def allreduce_max(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def bcast_int(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([int(x)], dtype=torch.int64)
    dist.broadcast(t, 0)
    return int(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def kg_energy(u, v, m):
    from oracle import diagnostics as D
    e = D.kg(u, v, m, np.ones_like(u), (CFG["L"], CFG["L"]))
    return float(e[0] + e[1] + e[2])


def cpu_parity_leg(k, traj, vel):
    """The FP64 oracle (C++/OpenMP restatement of the reference) runs
    trajectory 0 of the batch through the whole job (5999 steps, 50
    snapshots). Its wall time is the CPU baseline; its snapshots are the
    parity reference for the same trajectory of the end-to-end job (traj, vel:
    that job's snapshots of trajectory 0)."""
    from oracle import oracle as O
    seed, u0, v0, m, c = batch_fields(1, 0)[0]
    t0 = time.perf_counter()
    otraj, ovel = O.run(oracle_problem(k, seed=seed), u0, v0, m, c)
    secs = time.perf_counter() - t0
    steps = CFG["nt"] - 1
    rate = CFG["n"] ** 2 * steps / secs
    errs = [float(np.linalg.norm(traj[i] - otraj[i]) / np.linalg.norm(otraj[i])) for i in range(CFG["ns"])]
    e0 = kg_energy(otraj[0], ovel[0], m)
    parity = {"rel_l2_final": errs[-1], "rel_l2_max_snapshot": max(errs),
              "energy_drift": abs(kg_energy(traj[-1], vel[-1], m) - e0) / abs(e0),
              "energy_drift_oracle": abs(kg_energy(otraj[-1], ovel[-1], m) - e0) / abs(e0),
              "traj": 0, "steps": steps, "k": k, "bound": 1e-5,
              "against": "FP64 oracle (CGS re-orthogonalisation), final snapshot = state after step 5880"}
    cpu = {"value": rate, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
           "sample": f"trajectory 0 of the batch, 300^2, the whole job ({steps} steps, 50 snapshots) in "
                     f"{secs:.1f} s (FP64 oracle, CGS re-orthogonalisation, OpenMP over grid points)"}
    return cpu, parity


def _ref_spec(k, nt, ns, T):
    """The attributes oracle/ref_kg.py reads from a problem (no engine Spec)."""
    from types import SimpleNamespace
    n, L = CFG["n"], CFG["L"]
    return SimpleNamespace(dim=2, nx=n, ny=n, nz=1, Lx=L, Ly=L, Lz=L, shape=(n, n), n=n * n, k=k, nt=nt, ns=ns,
                           T=T, dt=T / nt)


def reference_device_path(k, steps=50):
    """The reference's own per-trajectory FP64 GPU path (device/include/
    kg_single.cuh step with its cuBLAS/cuSPARSE/cuSOLVER Lanczos matrix
    functions), compiled from its sources into oracle/_ref where the reference
    checkout was present at build time: trajectory 0 of the batch's 300^2 grid
    (the reference steps trajectories one at a time), dt = 0.005, Krylov
    dimension k, `steps` steps timed with CUDA events around its step loop
    after a short warm-up run. Reported beside the CPU baseline, not as the
    line's value."""
    from oracle import ref_kg
    if not ref_kg.available():
        return {"unavailable": "oracle/_ref/libref_kg.so not built (needs the reference checkout at build time)"}
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no GPU"}
        gpu = torch.cuda.get_device_name(0)
    except Exception as ex:  # torch without CUDA
        return {"unavailable": f"no GPU ({ex})"}
    seed, u0, v0, m, c = batch_fields(1, 0)[0]
    for nt in (3, steps + 1):  # a warm-up run, then the timed run
        spec = _ref_spec(k, nt, 1, nt * 0.005)
        _, _, ms = ref_kg.run(spec, u0, v0, m, 0)
    return {"value": spec.n * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps, "dtype": "f64",
            "gpu": gpu, "workload": f"trajectory 0 of the batch, 300^2, dt=0.005, k={k}, {steps} steps",
            "source": "device/include/kg_single.cuh step compiled from the reference's sources (oracle/_ref)"}


def run_reference(args, ws, rank, budget_s=150.0):
    """--impl reference: the FP64 CPU restatement of the reference algorithm at
    the same k and configuration as the engine's line. One step = one time
    step of the first B' trajectories of the batch (stateful, so no per-call
    setup is timed); B' = 64 unless --steps would run past about budget_s
    seconds, then fewer. Under torchrun only rank 0 runs. Nothing of the
    engine is imported: inputs come from the numpy-only field generators and
    the coefficients from the oracle's restatement of the reference."""
    if rank != 0:
        return 0
    k = K_HEADLINE
    # the reference's device path first: its step is bound by host round trips,
    # so it is timed before the oracle's OpenMP threads occupy the host cores
    try:
        dev = reference_device_path(k)
    except Exception as ex:  # reported, never fatal to the CPU line
        dev = {"unavailable": f"{type(ex).__name__}: {ex}"}
    from oracle import oracle as O
    fields = batch_fields(CFG["batch"], 0)
    n = CFG["n"] ** 2
    B = len(fields)
    steppers = [O.RealStepper(oracle_problem(k, seed=seed), u0, v0, m, c) for seed, u0, v0, m, c in fields]

    def one_step():
        t0 = time.perf_counter()
        for st in steppers:
            st.advance(1)
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        one_step()
    per_traj = one_step() / B
    keep = max(1, min(B, int(budget_s / max(args.steps * per_traj, 1e-9))))
    for st in steppers[keep:]:
        st.close()
    steppers = steppers[:keep]
    B = keep
    ts = [one_step() for _ in range(args.steps)]
    for st in steppers:
        st.close()
    total = sum(ts)
    value = B * n * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded kink/Gaussian u0, m = 1 + 0.2 GRF(k^-3))",
        "config": workload_config(k, ws, CFG["batch"]),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
                         "sample": f"{args.steps} timed steps of {B} of the 64 trajectories (FP64, CGS "
                                   "re-orthogonalisation, OpenMP over grid points)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    line["reference_device_path"] = dev
    print(json.dumps(line), flush=True)
    return 0


SERVE_RATES_HZ = (2.0, 8.0, 32.0, 128.0)
SERVE_WINDOW_S = 4.0  # arrivals span about this long at each rate
SERVE_REQUESTS = (12, 64)  # fewest and most requests of one rate's stream


def _serve_once(serve, reqs, budget, ws):
    """Serve this rank's requests; the line's row aggregates every rank's
    (grid-point-steps over the longest wall time, latencies of all requests)."""
    for r in reqs:
        r.t_admit, r.t_done, r.slot, r.traj = float("nan"), float("nan"), -1, None
    barrier(ws)
    if reqs:
        srv = serve.Server(serve.default_classes(reqs, max_slots=32), chunk=20, memory_budget=budget)
        st = srv.run(reqs, timeout_s=600)
        srv.close()
    else:
        st = serve.ServeStats(completed=0, wall_s=0.0, gp_steps=0)
    stats = [st]
    if ws > 1:
        import torch.distributed as dist
        stats = [None] * ws
        dist.all_gather_object(stats, st)
    row = serve.merge_stats(stats) if ws > 1 else st.summary()
    row.update({"requests": sum(s_.completed for s_ in stats),
                "classes": sorted({r.cls for r in reqs}), "gp_steps": sum(s_.gp_steps for s_ in stats)})
    return row


def serving_leg(ws=1, rank=0, rates=SERVE_RATES_HZ, window_s=SERVE_WINDOW_S, steps=(500, 5000), seed=5,
                budget_gib=8.0):
    """The serving mix (requests uniform over KG 2-D 64^2-300^2, NLSE 2-D
    64^2-256^2, KG 3-D 64^3-160^3 and phi^4 2-D, 500-5000 steps each, Poisson
    arrivals) at each rate of `rates` per GPU: latency percentiles (arrival to
    last snapshot on the host) and aggregate throughput (all requests'
    grid-point-steps over the run's wall time). One stream of 64 requests per
    GPU is drawn with Poisson arrivals at 1 Hz per GPU; the stream of rate r is
    its first rate x window_s requests per GPU (at least 12, at most 64) with
    the arrival times divided by r, so the higher rates keep the servers loaded
    for most of their run. With several GPUs each rate's stream is placed on
    them by grid-point-steps (serve.partition, largest first) and every rank
    serves its share with its own server (weak scaling: the stream grows with
    the GPUs). "saturated" serves the whole stream arriving at once: the
    throughput ceiling of this mix on these servers. Admission by an 8 GiB
    device-memory budget per GPU shared by its class pools; page-locked client
    snapshot buffers."""
    from nlsb200 import serve
    budget = int(budget_gib * (1 << 30))
    out = {"rates": [], "arrival_window_s": window_s, "steps_per_request": list(steps), "unit": UNIT,
           "memory_budget_bytes": budget, "snapshots_per_request": 5, "n_gpus": ws,
           "placement": "greedy by grid-point-steps" if ws > 1 else "one GPU"}
    plans = serve.mixed_plans(SERVE_REQUESTS[1] * ws, float(ws), seed=seed, steps=steps)
    base = {pl.rid: pl.arrival for pl in plans}
    built = {}

    def mine(sub):
        part = serve.partition(sub, ws)[rank]
        for pl in part:
            if pl.rid not in built:
                built[pl.rid] = serve.build_request(pl, ns=5, pinned=True)
        return [built[pl.rid] for pl in part]

    for rate in rates:
        count = int(min(max(round(rate * window_s), SERVE_REQUESTS[0]), SERVE_REQUESTS[1])) * ws
        reqs = mine(plans[:count])
        for r in reqs:
            r.arrival = base[r.rid] / rate
        row = _serve_once(serve, reqs, budget, ws)
        row["rate_hz"] = rate
        out["rates"].append(row)
    reqs = mine(plans)
    for r in reqs:
        r.arrival = 0.0
    out["saturated"] = _serve_once(serve, reqs, budget, ws)
    built.clear()
    return out


def other_configs_leg(steps=20, reps=3):
    """The other batched configurations, timed the same way as the headline
    (inputs resident, graph replay, CUDA events on the pool stream, median of
    `reps` blocks of `steps` steps after 3 warm-up steps):
      - NLSE 2-D SS2, 128 x 200^2 on [-10,10]^2, dt = 1e-3, k = 12, complex64;
      - KG 3-D Gautschi, 40 x 220^3 on [-10,10]^3, dt = 0.01, k = 10, FP32.
    The fields of NLSE trajectory i are those of seed i % 16, of 3-D
    trajectory i those of seed i % 4 (the shapes and distributions of the
    configuration; fewer distinct fields keep the host-side generation short).
    Each entry carries the roofline of its Lanczos pass: 24 algorithmic bytes
    per grid point (three vectors of 8 B for complex64 with one sequence, of
    4 B for each of the two real sequences), passes j = 2..k-2 back to back."""
    import nlsb200 as nl
    from nlsb200 import workloads as W
    from nlsb200.solver import FP32, KG_GAUTSCHI, NLSE_SS2, Pool
    peak, peak_kind = hbm_peak()
    out = {}
    for name in ("nlse2d_200_b128", "kg3d_220_b40"):
        cfg = W.CONFIGS[name]
        n, B, k = cfg["n"], cfg["batch"], cfg["k"]
        dim = 3 if name.startswith("kg3d") else 2
        distinct = 16 if dim == 2 else 4
        if dim == 2:
            base = [W.nlse_case(n, cfg["L"], cfg["T"], cfg["nt"], cfg["ns"], k=k, seed=i, precision=FP32)
                    for i in range(distinct)]
            method = NLSE_SS2
        else:
            base = [W.kg_case(n, cfg["L"], cfg["T"], cfg["nt"], cfg["ns"], k=k, seed=i, dim=3, precision=FP32)
                    for i in range(distinct)]
            method = KG_GAUTSCHI
        if dim == 3:
            # one snapshot (the initial state): at the configuration's cadence
            # (every 250 steps) the timed steps hold no snapshot step either
            for sp, *_ in base:
                sp.ns = 1
        # every trajectory's host snapshot buffer is one shared page-locked array
        # (the timing leg reads no result back)
        sp0 = base[0][0]
        shared_traj = nl.pinned_empty((sp0.ns,) + sp0.shape, np.complex128 if dim == 2 else np.float64)
        shared_vel = None if dim == 2 else nl.pinned_empty((sp0.ns,) + sp0.shape)
        cases = [base[i % distinct] for i in range(B)]
        pts = ((n + 31) // 32 * 32) * n * (n if dim == 3 else 1)
        # NLSE 2-D: 25-row pass segments, 20-row final tiles (12 / 16 / 20 / 25 rows measured 0.537 /
        # 0.543 / 0.534 / 0.570 ms per step); 3-D: 88-plane segments (the default)
        pool = Pool(method, dim, k, FP32, capacity_points=B * (pts + 256), max_slots=B,
                    segment=25 if dim == 2 else None, final_segment=20 if dim == 2 else None)
        for cs in cases:
            assert pool.admit(*cs, traj=shared_traj, vel=shared_vel) is not None
        pool.step(3)
        pool.sync()
        ms = statistics.median([pool.step_timed(steps) / steps for _ in range(reps)])
        pass_ms, ppts = pool.time_passes(2, k - 2, 5)
        pool.close()
        npts = B * n ** dim
        achieved = 24 * ppts / (pass_ms / 1e3) / 1e9
        out[name] = {
            "workload": (f"NLSE 2-D SS2, {B} x {n}^2 on [-10,10]^2, dt=1e-3, k={k}, complex64" if dim == 2 else
                         f"KG 3-D Gautschi, {B} x {n}^3 on [-10,10]^3, dt=0.01, k={k}, FP32"),
            "ms_per_step": ms, "value": npts / (ms / 1e3), "unit": UNIT, "steps": steps * reps,
            "pass_roofline": {"kernel": "k2_lanczos1_c32" if dim == 2 else "k3_lanczos_f32",
                              "launch_ms": pass_ms, "achieved": achieved, "peak": peak, "unit": "GB/s",
                              "frac": achieved / peak, "peak_kind": peak_kind},
        }
        del base, cases, shared_traj, shared_vel
    return out


def run_small(args, lrank):
    """--small: --batch trajectories (default 16) of the same workload (--k,
    default the benchmark's; --seg-row segments), warmup + steps only; the case the ncu captures profile
    (16: ~0.2 GB, 64: ~0.7 GB on the GPU, both above the 126 MB L2)."""
    import nlsb200 as nl
    from nlsb200 import workloads as W
    from nlsb200.solver import FP32, KG_GAUTSCHI, Pool
    nl.lib().nls_set_device(lrank)
    B, k = args.batch, args.k
    dim = 3 if args.dim3 else 2
    method = KG_GAUTSCHI
    if args.nlse:
        # NLSE 2-D SS2 boxes of 200^2 on [-10,10]^2, dt = 1e-3, k = 12 (the batched NLSE configuration's shape)
        from nlsb200.solver import NLSE_SS2
        method, k = NLSE_SS2, 12
        cases = [W.nlse_case(200, 10.0, T=2.0, nt=2000, ns=100, k=k, seed=i, precision=FP32) for i in range(B)]
        cap = sum(((s.nx + 31) // 32 * 32) * s.ny for s, *_ in cases) + 256 * B
    elif dim == 3:
        # KG 3-D Gautschi boxes of dim3^3 on [-10,10]^3, dt = 0.01, 40 snapshots
        cases = [W.kg_case(args.dim3, 10.0, T=100.0, nt=10000, ns=40, k=k, seed=i, dim=3, precision=FP32)
                 for i in range(B)]
        cap = sum(((s.nx + 31) // 32 * 32) * s.ny * s.nz for s, *_ in cases) + 256 * B
    else:
        cases = make_batch(B, 0, k)
        cap = sum(((s.nx + 31) // 32 * 32) * s.ny for s, *_ in cases) + 256 * B
    pool = Pool(method, dim, k, FP32, capacity_points=cap, max_slots=B, segment=args.seg,
                final_segment=args.fseg if dim == 2 else None)
    for cs in cases:
        assert pool.admit(*cs) is not None
    pool.step(args.warmup)
    ms = pool.step_timed(args.steps)
    pool.sync()
    pass_ms, _ = pool.time_pass(2, 20)
    chain_ms = pool.time_passes(2, k - 2, 10)[0] if k >= 4 else None
    print(json.dumps({"small": True, "method": int(method), "dim": dim, "n": cases[0][0].nx, "batch": B, "k": k, "seg": args.seg,
                      "fseg": args.fseg,
                      "ms_per_step": ms / args.steps,
                      "pass_ms": pass_ms, "pass_chain_ms": chain_ms,
                      "kernels_per_step": pool.kernels_per_step()}), flush=True)
    pool.close()
    return 0


def timed_blocks(pool, steps, ws, target_s=TIMED_REGION_S, max_blocks=200):
    """Blocks of exactly `steps` steps, each bracketed by a barrier and a device
    sync and timed with CUDA events on the pool's stream (max over ranks),
    repeated until they add up to about target_s; returns the block times."""
    times = []
    while True:
        pool.sync()
        barrier(ws)
        ms = allreduce_max(pool.step_timed(steps), ws)
        times.append(ms)
        nblk = len(times)
        if nblk >= max_blocks or bcast_int(int(sum(times) >= 1e3 * target_s), ws):
            break
    pool.sync()
    barrier(ws)
    return times


def run_ours(args, ws, rank, lrank):
    import nlsb200 as nl
    from nlsb200 import autotune
    from nlsb200.solver import FP32, KG_GAUTSCHI, Pool

    if args.small:
        return run_small(args, lrank)
    nl.lib().nls_set_device(lrank)
    B = CFG["batch"]
    k = K_HEADLINE
    tuning = {}
    if rank == 0:
        # the live re-check of k: the reference leaves T[k-1,k-1] = 0, so its
        # result converges only algebraically in k; the autotuner accepts k
        # when 10 probe steps stay within 5e-6 of k = 24
        probe = make_batch(1, 0, 16)[0]
        k_auto, kreport = autotune.choose_k(*probe, candidates=tuple(range(8, 17)), k_ref=24, steps=10, tol=5e-6)
        tuning.update({"k_autotune": k_auto, "k_autotune_err": kreport, "k_used": k})
    cases = make_batch(B, rank, k)
    n = cases[0][0].n
    cap = sum(((s.nx + 31) // 32 * 32) * s.ny for s, *_ in cases) + 256 * B

    # the final pass sums nothing across tiles and keeps its own 25-row tiles
    # (one wave of warps for the batch; 12 / 16 / 20 / 25 / 30 rows measured
    # 0.346 / 0.345 / 0.358 / 0.340 / 0.346 ms per step with 28-row passes)
    # (more warps than the passes' segments give it)
    def make_pool(seg):
        return Pool(KG_GAUTSCHI, 2, k, FP32, capacity_points=cap, max_slots=B, segment=seg, final_segment=FINAL_ROWS)

    def admit_all(pool):
        for cs in cases:
            assert pool.admit(*cs) is not None

    # 25 rows: 12 segments x 3 strips x 2 sequences x 32 trajectories per group
    # = 2304 warps, one wave of 16 warps on each of the 148 SMs
    seg, seg_times = autotune.choose_segment(make_pool, admit_all, candidates=(16, 25, 28, 32), steps=6)
    seg = bcast_int(seg, ws)  # every rank runs rank 0's tiling
    tuning.update({"segment_rows": seg, "final_segment_rows": FINAL_ROWS, "segment_ms": seg_times})
    pool = make_pool(seg)
    admit_all(pool)
    pool.step(args.warmup)
    pool.sync()
    barrier(ws)
    with Clocks(lrank) as clk:
        blocks = timed_blocks(pool, args.steps, ws)
    ms = statistics.median(blocks)
    value = ws * B * n * args.steps / (ms / 1e3)
    kernels = pool.kernels_per_step()
    # dominant kernel: the Lanczos passes j = 2 .. k-2 (the plain form of
    # k2_lanczos1_f32c), launched back to back as the step issues them, CUDA
    # events on the pool stream; and pass j = 2 forked and joined around every
    # launch (a launch in isolation), for reference
    pass_ms, pts = pool.time_passes(2, k - 2, 10)
    pass_iso_ms, _ = pool.time_pass(2, 20)
    peak, peak_kind = hbm_peak()
    pass_bytes = pass_bytes_per_gp() * pts
    achieved = pass_bytes / (pass_ms / 1e3) / 1e9
    step_bytes = step_bytes_per_gp(k) * B * n
    pool.close()

    # end to end through the public API: the configuration's complete job
    # (nt = 6000: steps 1 .. 5999, 50 snapshots every 120 steps) with admission
    # (H2D of every input), the steps, every snapshot's D2H and the release
    e_steps = CFG["nt"] - 1
    ecases = make_batch(B, rank, k)
    # page-locked input and snapshot buffers, allocated before the timed region
    pinned = []
    for spec, u0, v0, m, c in ecases:
        pu, pv, pm = (nl.pinned_empty(spec.shape) for _ in range(3))
        pu[...] = u0
        pv[...] = v0
        pm[...] = m
        tr = nl.pinned_empty((spec.ns,) + spec.shape)
        ve = nl.pinned_empty((spec.ns,) + spec.shape)
        pinned.append((spec, pu, pv, pm, c, tr, ve))
    epool = make_pool(seg)
    barrier(ws)
    t0 = time.perf_counter()
    slots = [epool.admit(spec, pu, pv, pm, c, traj=tr, vel=ve)
             for spec, pu, pv, pm, c, tr, ve in pinned]
    epool.step(e_steps)
    epool.sync()
    outs = [epool.release(s) for s in slots]
    e_time = allreduce_max(time.perf_counter() - t0, ws)
    epool.close()
    d2h = sum(2 * s.ns * s.n * 8 for s, *_ in ecases)  # every snapshot frame (u, v) in FP64
    h2d = sum(3 * s.n * 8 for s, *_ in ecases)  # u0, v0, m in FP64 (c == 1 is not sent)
    e2e = {"value": ws * B * n * e_steps / e_time, "unit": UNIT,
           "h2d_bytes_per_step": h2d / e_steps, "d2h_bytes_per_step": d2h / e_steps,
           "note": "the configuration's complete job (64 x 300^2, 6000 steps, 50 snapshots) through "
                   "nlsb200.Pool: admit (H2D of every input from page-locked memory), 5999 steps, "
                   "every snapshot's D2H into page-locked memory, release; bytes amortised per step"}
    traj0, vel0 = np.array(outs[0].traj), np.array(outs[0].vel)
    del outs, pinned

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded kink/Gaussian u0, m = 1 + 0.2 GRF(k^-3))",
        "config": workload_config(k, ws, B),
        "timed_blocks": {"blocks": len(blocks), "steps_per_block": args.steps,
                         "median_ms": ms, "min_ms": min(blocks), "max_ms": max(blocks),
                         "total_s": sum(blocks) / 1e3},
        "tuning": tuning,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": TRAFFIC_BYTES_PER_POINT_PASS * pts,
                     "peak_kind": peak_kind,
                     "kernel": f"k2_lanczos1_f32c (2-D FP32 Lanczos passes j=2..{k - 2}, in the step's order)",
                     "bytes_per_launch": pass_bytes, "launch_ms": pass_ms,
                     "launch_ms_isolated": pass_iso_ms,
                     "frac_isolated": pass_bytes / (pass_iso_ms / 1e3) / 1e9 / peak},
        "step_roofline": {"algorithmic_bytes_per_gp_step": step_bytes_per_gp(k),
                          "achieved_GBps": step_bytes * args.steps / (ms / 1e3) / 1e9,
                          "frac": step_bytes * args.steps / (ms / 1e3) / 1e9 / peak},
        "e2e": e2e,
        "gpu_launches": kernels * args.steps * len(blocks),
        "kernels_per_step": kernels,
        "clocks": clk.summary(),
    }
    if not args.no_serve:
        line["serving"] = serving_leg(ws, rank)
    if ws == 1 and not args.no_other:
        line["other_configs"] = other_configs_leg()
    if ws == 1 and rank == 0 and not args.no_cpu:
        line["cpu_baseline"], line["parity"] = cpu_parity_leg(k, traj0, vel0)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def spawn_ranks(n):
    """--gpus N without a launcher: start the N ranks through
    torch.distributed.run on 127.0.0.1 with this command line and return
    their exit status (rank 0 prints the line)."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle baseline and parity leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-mix leg")
    ap.add_argument("--no-other", action="store_true", help="skip the NLSE 2-D and KG 3-D batched configurations")
    ap.add_argument("--small", action="store_true",
                    help="profiling case of --batch trajectories (no autotune, e2e or CPU leg)")
    ap.add_argument("--batch", type=int, default=16, help="trajectories of the --small case")
    ap.add_argument("--seg", type=int, default=32, help="segment rows (planes in 3-D) of the --small case")
    ap.add_argument("--fseg", type=int, default=0, help="2-D final-pass segment rows of the --small case (0: --seg)")
    ap.add_argument("--k", type=int, default=K_HEADLINE, help="Krylov dimension of the KG --small case")
    ap.add_argument("--nlse", action="store_true", help="--small case as NLSE 2-D SS2 boxes of 200^2 (k = 12)")
    ap.add_argument("--dim3", type=int, default=0,
                    help="--small case as KG 3-D boxes of DIM3^3 points (0: the 2-D 300^2 workload)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus < 1:
        print(f"bench.py: --gpus must be at least 1 (got {args.gpus})", file=sys.stderr)
        return 2
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return spawn_ranks(args.gpus)
    ws, rank, lrank = dist_init()
    if ws != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but {ws} rank(s) joined (WORLD_SIZE={ws}); "
              "launch one process per GPU", file=sys.stderr)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return 2
    try:
        if args.impl == "reference":
            return run_reference(args, ws, rank)
        return run_ours(args, ws, rank, lrank)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
