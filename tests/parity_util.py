"""Shared helpers of the parity tests: run the FP64 oracle on a Spec."""
import numpy as np

from oracle import oracle as O


def oracle_problem(spec, reorth=True, max_steps=0):
    prm = spec.oracle_params()
    return O.Problem(dim=spec.dim, nx=spec.nx, ny=spec.ny, nz=spec.nz if spec.dim == 3 else 1,
                     Lx=spec.Lx, Ly=spec.Ly, Lz=spec.Lz, T=spec.T, nt=spec.nt, ns=spec.ns,
                     k=prm["k"], method=spec.method, sewi_variant=spec.sewi_variant,
                     reorth=int(reorth), max_steps=max_steps, p1=prm["p1"], q1=prm["q1"],
                     p3=prm["p3"], q3=prm["q3"], rm=prm["rm"], r0=prm["r0"], seed=spec.seed,
                     nonlinearity=prm["nonlinearity"])


def run_oracle(spec, u0, v0, m, c, reorth=True):
    if c is None:
        c = np.ones(spec.shape)
    return O.run(oracle_problem(spec, reorth), u0, v0, m, c)
