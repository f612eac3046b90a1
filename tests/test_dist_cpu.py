"""The multi-rank plumbing of bench.py on CPU: two gloo ranks over 127.0.0.1.

bench.py shards trajectories across ranks with no data-path collective; the
process group carries only the barrier, rank 0's choices (Krylov dimension,
segment rows) and the max over ranks of the device timings. This runs those
helpers in two real processes and checks what each rank sees.
"""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import json, os, sys, time
sys.path.insert(0, os.environ["NLS_ROOT"])
sys.path.insert(0, os.path.join(os.environ["NLS_ROOT"], "nlsolvers-datagen_b200"))
import bench
ws, rank, lrank = bench.dist_init()
out = {"ws": ws, "rank": rank}
out["max"] = bench.allreduce_max(0.5 + rank, ws)
out["k"] = bench.bcast_int(9 if rank == 0 else 12, ws)
bench.barrier(ws)
cases = bench.make_batch(2, rank, 10)
out["u0"] = [float(abs(c[1]).sum()) for c in cases]
import hashlib
out["m"] = [hashlib.sha1(c[3].tobytes()).hexdigest() for c in cases]
class A:
    steps, warmup, gpus = 3, 3, ws
t0 = time.perf_counter()
out["ref_rc"] = bench.run_reference(A, ws, rank) if rank == 1 else 0
out["ref_s"] = time.perf_counter() - t0
import torch.distributed as dist
dist.destroy_process_group()
print("RESULT " + json.dumps(out), flush=True)
"""


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_and_reduce():
    port = _port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE="2",
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), NLS_ROOT=ROOT)
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    res = []
    for p in procs:
        out, err = p.communicate(timeout=240)
        assert p.returncode == 0, err[-2000:]
        line = [x for x in out.splitlines() if x.startswith("RESULT ")][-1]
        res.append(json.loads(line[7:]))
    r0, r1 = sorted(res, key=lambda d: d["rank"])
    assert r0["ws"] == r1["ws"] == 2
    assert r0["max"] == r1["max"] == 1.5          # max over ranks of the timings
    assert r0["k"] == r1["k"] == 9                 # every rank takes rank 0's choice
    # the shards are different trajectories (seeded by rank), not copies
    assert r0["u0"] != r1["u0"] and r0["m"] != r1["m"]
    # the reference arm runs on rank 0 only: rank 1 returns 0 without work
    assert r1["ref_rc"] == 0 and r1["ref_s"] < 1.0
