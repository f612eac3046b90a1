#!/usr/bin/env python
"""Benchmark of the batched Lanczos exponential integrator (one JSON line).

Workload (the headline batched configuration): 64 nonlinear Klein-Gordon
trajectories u_tt = Lap u - m u^3 on [-15,15]^2, 300 x 300 grid (incl. ghost
ring), Gautschi step with a k-step Lanczos cos / sinc^2 filter (k picked by the
project autotuner in 8..16), dt = 0.005, nt = 6000, 50 snapshots, FP32 Krylov
basis + compensated FP32 fields. A "step" is one time step of the whole batch.
Inputs are seeded synthetic fields (kink/Gaussian mixtures, m = 1 + 0.2 GRF).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun, one process per GPU): every rank steps its own 64 trajectories
(weak scaling, no data-path collective); the step time is the max over ranks.
--impl reference times the reference algorithm's CPU restatement (the FP64
oracle; the reference itself has no CPU path) on the host cores, rank 0 only,
and reports beside it the reference's own per-trajectory FP64 GPU path,
compiled from its sources, on one trajectory of the same grid.
"""
from __future__ import annotations

import argparse
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
FALLBACK_HBM = 6650.0


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


def make_batch(B, rank, k, nt=None, ns=None, T=None):
    from nlsb200 import workloads as W
    cases = []
    for i in range(B):
        spec, u0, v0, m, c = W.kg_case(CFG["n"], CFG["L"], T or CFG["T"], nt or CFG["nt"],
                                       ns or CFG["ns"], k=k, seed=1000 * rank + i,
                                       kinks=(i % 2 == 0))
        cases.append((spec, u0, v0, m, c))
    return cases


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


def cpu_oracle_rate(cases, budget_s=12.0):
    """FP64 oracle (C++/OpenMP restatement of the reference) on one trajectory of
    the batch for a bounded number of pure steps; returns gp-steps/s."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle import oracle as O
    from parity_util import oracle_problem
    spec, u0, v0, m, c = cases[0]
    st = O.RealStepper(oracle_problem(spec, reorth=True), u0, v0, m, c)
    st.advance(1)
    t0 = time.perf_counter()
    st.advance(2)
    per = (time.perf_counter() - t0) / 2
    steps = max(2, min(spec.nt - 4, int(budget_s / max(per, 1e-4))))
    t0 = time.perf_counter()
    st.advance(steps)
    dt = time.perf_counter() - t0
    st.close()
    return spec.n * steps / dt, steps, dt, O.num_threads()


def reference_device_path(steps=50):
    """The reference's own per-trajectory FP64 GPU path (device/include/
    kg_single.cuh step with its cuBLAS/cuSPARSE/cuSOLVER Lanczos matrix
    functions), compiled from its sources into oracle/_ref where the reference
    checkout was present at build time: one trajectory of the batch's 300^2
    grid (the reference steps trajectories one at a time), dt = 0.005, k = 10,
    `steps` steps timed with CUDA events around its step loop after a short
    warm-up run. Reported beside the CPU baseline, not as the line's value."""
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
    for nt in (3, steps + 1):  # a warm-up run, then the timed run
        spec, u0, v0, m, _ = make_batch(1, 0, 10, nt=nt, ns=1, T=nt * 0.005)[0]
        _, _, ms = ref_kg.run(spec, u0, np.zeros_like(u0), m, 0)
    return {"value": spec.n * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps, "dtype": "f64",
            "gpu": gpu, "workload": f"one 300^2 trajectory of the batch, dt=0.005, k=10, {steps} steps",
            "source": "device/include/kg_single.cuh step compiled from the reference's sources (oracle/_ref)"}


def run_reference(args, ws, rank, budget_s=150.0):
    """--impl reference: the FP64 CPU restatement of the reference algorithm
    (its own k = 10 for kg_gautschi_2d_dev). One step = one time step of the
    first B' trajectories of the batch (stateful, so no per-call setup is
    timed); B' = 64 unless --steps would run past about budget_s seconds, then
    fewer. Under torchrun only rank 0 runs."""
    if rank != 0:
        return 0
    # the reference's device path first: its step is bound by host round trips,
    # so it is timed before the oracle's OpenMP threads occupy the host cores
    try:
        dev = reference_device_path()
    except Exception as ex:  # reported, never fatal to the CPU line
        dev = {"unavailable": f"{type(ex).__name__}: {ex}"}
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle import oracle as O
    from parity_util import oracle_problem
    k = 10
    cases = make_batch(CFG["batch"], 0, k)
    n = cases[0][0].n
    B = len(cases)
    steppers = [O.RealStepper(oracle_problem(spec, reorth=True), u0, v0, m, c)
                for spec, u0, v0, m, c in cases]

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
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded kink/Gaussian u0, m = 1 + 0.2 GRF(k^-3))",
        "config": {"workload": "KG 2-D Gautschi batch, 64 x 300^2 on [-15,15]^2, dt=0.005, k=10",
                   "global_batch": B, "grid": [CFG["n"], CFG["n"]], "k": k},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
                         "sample": f"{args.steps} timed steps of {B} of the 64 trajectories (FP64, CGS re-orthogonalisation, OpenMP over grid points)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    line["reference_device_path"] = dev
    print(json.dumps(line), flush=True)
    return 0


def serving_leg(count=24, rate_hz=8.0, steps=(200, 600), seed=5):
    """The serving mix (requests uniform over KG 2-D 64^2-300^2, NLSE 2-D
    64^2-256^2, KG 3-D 64^3-160^3 and phi^4 2-D; Poisson arrivals), shortened
    to `steps` per request so that it runs in seconds: latency percentiles
    (arrival to last snapshot on the host) and aggregate throughput."""
    from nlsb200 import serve
    reqs = serve.mixed_requests(count, rate_hz, seed=seed, steps=steps)
    srv = serve.Server(serve.default_classes(reqs, max_slots=16), chunk=10)
    st = srv.run(reqs, timeout_s=300)
    srv.close()
    out = st.summary()
    out.update({"requests": count, "rate_hz": rate_hz, "steps_per_request": list(steps),
                "classes": sorted({r.cls for r in reqs}), "unit": UNIT})
    return out


def run_small(args, lrank):
    """--small: --batch trajectories (default 16) of the same workload (k=10,
    32-row segments), warmup + steps only; the case the ncu captures profile
    (16: ~0.2 GB, 64: ~0.7 GB on the GPU, both above the 126 MB L2)."""
    import nlsb200 as nl
    from nlsb200 import workloads as W
    from nlsb200.solver import FP32, KG_GAUTSCHI, Pool
    nl.lib().nls_set_device(lrank)
    B, k = args.batch, 10
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
    print(json.dumps({"small": True, "method": int(method), "dim": dim, "n": cases[0][0].nx, "batch": B, "k": k, "seg": args.seg,
                      "fseg": args.fseg,
                      "ms_per_step": ms / args.steps,
                      "pass_ms": pass_ms, "kernels_per_step": pool.kernels_per_step()}), flush=True)
    pool.close()
    return 0


def run_ours(args, ws, rank, lrank):
    import nlsb200 as nl
    from nlsb200 import autotune
    from nlsb200.solver import FP32, KG_GAUTSCHI, Pool

    if args.small:
        return run_small(args, lrank)
    nl.lib().nls_set_device(lrank)
    B = CFG["batch"]
    # k by the a-posteriori Krylov error estimate on rank 0's first trajectory
    probe = make_batch(1, 0, 16)[0]
    k = None
    kreport = {}
    if rank == 0:
        # the reference leaves T[k-1,k-1] = 0, so its result converges only
        # algebraically in k; accept k when 10 probe steps stay within 5e-6 of k = 24
        k, kreport = autotune.choose_k(*probe, candidates=tuple(range(8, 17)), k_ref=24,
                                       steps=10, tol=5e-6)
    k = bcast_int(k if k is not None else 0, ws)
    cases = make_batch(B, rank, k)
    n = cases[0][0].n
    cap = sum(((s.nx + 31) // 32 * 32) * s.ny for s, *_ in cases) + 256 * B

    # the final pass sums nothing across tiles and keeps its own 16-row tiles
    # (more warps than the passes' segments give it)
    def make_pool(seg):
        return Pool(KG_GAUTSCHI, 2, k, FP32, capacity_points=cap, max_slots=B, segment=seg, final_segment=16)

    def admit_all(pool):
        for cs in cases:
            assert pool.admit(*cs) is not None

    # 25 rows: 12 segments x 3 strips x 2 sequences x 32 trajectories per group
    # = 2304 warps, one wave of 16 warps on each of the 148 SMs
    seg, seg_times = autotune.choose_segment(make_pool, admit_all, candidates=(16, 25, 28, 32), steps=6)
    seg = bcast_int(seg, ws)  # every rank runs rank 0's tiling
    pool = make_pool(seg)
    admit_all(pool)
    pool.step(args.warmup)
    pool.sync()
    barrier(ws)
    with Clocks(lrank) as clk:
        ms = pool.step_timed(args.steps)
    pool.sync()
    ms = allreduce_max(ms, ws)
    barrier(ws)
    value = ws * B * n * args.steps / (ms / 1e3)
    kernels = pool.kernels_per_step()
    # dominant kernel: Lanczos pass (j = 2), timed alone with CUDA events
    pass_ms, pts = pool.time_pass(2, 20)
    peak, peak_kind = hbm_peak()
    pass_bytes = pass_bytes_per_gp() * pts
    achieved = pass_bytes / (pass_ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "ncu_lanczos_pass_kg2d.md")
    if os.path.exists(tpath):
        for line in open(tpath):
            if line.startswith("traffic_bytes_per_point:"):
                traffic = float(line.split(":")[1]) * pts
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
    del outs

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded kink/Gaussian u0, m = 1 + 0.2 GRF(k^-3))",
        "config": {"workload": "KG 2-D Gautschi batch, 64 x 300^2 on [-15,15]^2, dt=0.005, nt=6000, ns=50",
                   "global_batch": B * ws, "per_gpu_batch": B, "grid": [CFG["n"], CFG["n"]],
                   "k": k, "k_autotune_err": kreport, "segment_rows": seg, "final_segment_rows": 16,
                   "segment_ms": seg_times, "parallelism": f"trajectory shards x{ws}",
                   "l2": "working set 0.6 GB per GPU >> 126 MB L2 (no flush needed)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": "k2_lanczos1_f32c (2-D FP32 Lanczos pass j=2)",
                     "bytes_per_launch": pass_bytes, "launch_ms": pass_ms},
        "step_roofline": {"algorithmic_bytes_per_gp_step": step_bytes_per_gp(k),
                          "achieved_GBps": step_bytes * args.steps / (ms / 1e3) / 1e9 * 1.0,
                          "frac": step_bytes * args.steps / (ms / 1e3) / 1e9 / peak},
        "e2e": e2e,
        "gpu_launches": kernels * args.steps,
        "kernels_per_step": kernels,
        "clocks": clk.summary(),
    }
    if ws == 1 and not args.no_serve:
        line["serving"] = serving_leg()
    if ws == 1 and rank == 0 and not args.no_cpu:
        rate, steps, secs, cores = cpu_oracle_rate(cases)
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": f"1 trajectory 300^2, {steps} steps in {secs:.1f} s (FP64 oracle, CGS re-orthogonalisation)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU oracle baseline")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-mix leg")
    ap.add_argument("--small", action="store_true",
                    help="profiling case of --batch trajectories (no autotune, e2e or CPU leg)")
    ap.add_argument("--batch", type=int, default=16, help="trajectories of the --small case")
    ap.add_argument("--seg", type=int, default=32, help="segment rows (planes in 3-D) of the --small case")
    ap.add_argument("--fseg", type=int, default=0, help="2-D final-pass segment rows of the --small case (0: --seg)")
    ap.add_argument("--nlse", action="store_true", help="--small case as NLSE 2-D SS2 boxes of 200^2 (k = 12)")
    ap.add_argument("--dim3", type=int, default=0,
                    help="--small case as KG 3-D boxes of DIM3^3 points (0: the 2-D 300^2 workload)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, lrank = dist_init()
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
