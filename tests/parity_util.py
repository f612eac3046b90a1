"""Shared helpers of the parity tests: run the FP64 oracle on a Spec.

The oracle's equation coefficients come from the oracle's own restatement of
the reference (oracle.reference_coefficients), overridden only by what the
test's Spec sets explicitly; nothing is read back from the product library.
"""
import numpy as np

from oracle import oracle as O


def oracle_params(spec):
    """k and nonlinearity coefficients for the oracle: the reference's values
    for spec.method, with every coefficient the Spec sets explicitly (k, p1,
    p3, rm; q1, q3, r0 and the nonlinearity kind always) taking precedence."""
    prm = O.reference_coefficients(spec.method, spec.dim, spec.nx, spec.Lx, spec.T / spec.nt)
    if spec.k is not None:
        prm["k"] = spec.k
    for name in ("p1", "p3", "rm"):
        v = getattr(spec, name)
        if v is not None:
            prm[name] = float(v)
    prm["q1"], prm["q3"], prm["r0"] = float(spec.q1), float(spec.q3), float(spec.r0)
    prm["nonlinearity"] = int(spec.nonlinearity)
    return prm


def oracle_problem(spec, reorth=True, max_steps=0):
    prm = oracle_params(spec)
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
