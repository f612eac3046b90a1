"""Project autotuner: Krylov dimension k and march-segment length.

k is chosen a posteriori: one trajectory of the batch is advanced a few steps
with each candidate k and with a larger reference k on the engine itself; the
smallest k whose state differs from the reference by less than `tol` (rel-L2)
wins. The same k must then be used by any parity check (the oracle reruns with
the chosen k). The segment length only changes the tiling (rounding order), so
it is picked by timing a few steps of the full batch.
"""
from __future__ import annotations

import numpy as np

from .solver import Pool, Solver, Spec


def _probe(spec: Spec, u0, v0, m, c, k: int, steps: int):
    s = Spec(**{**spec.__dict__, "k": k, "nt": 2 * steps, "ns": 2, "T": spec.dt * 2 * steps})
    with Solver(s, u0, v0, m, c) as sol:
        sol.step(steps)
        traj, _ = sol.snapshots()
    return traj[1]


def choose_k(spec: Spec, u0, v0, m, c, candidates=(8, 9, 10, 12, 14, 16), k_ref=24,
             steps=20, tol=1e-8):
    """Smallest candidate k whose probe state matches the k_ref probe within tol."""
    ref = _probe(spec, u0, v0, m, c, k_ref, steps)
    nref = np.linalg.norm(ref)
    report = {}
    for k in sorted(candidates):
        got = _probe(spec, u0, v0, m, c, k, steps)
        err = float(np.linalg.norm(got - ref) / nref)
        report[k] = err
        if err < tol:
            return k, report
    return max(candidates), report


def choose_segment(make_pool, admit_all, candidates=(16, 32, 64), steps=4):
    """Time `steps` steps for each segment length on a fresh pool; fastest wins."""
    best, times = None, {}
    for seg in candidates:
        pool = make_pool(seg)
        admit_all(pool)
        pool.step(2)
        ms = pool.step_timed(steps)
        times[seg] = ms / steps
        pool.close()
        if best is None or times[seg] < times[best]:
            best = seg
    return best, times
