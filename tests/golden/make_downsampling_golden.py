"""Generate tests/golden/downsampling.npz from the reference's own Python
downsampling.

The reference's HDF5 aggregation downsamples every snapshot on the host with
scripts/downsampling.py:68-103 (downsample_interpolation, 2-D) and
scripts/downsampling.py:215-257 (downsample_interpolation_3d), called from
scripts/aggregate_single.py:61-76: linear RegularGridInterpolator on the
linspace(-L, L, n) grids of the source and of the target shape. The module
imports torch and matplotlib at the top, so this script parses the file and
executes only those two function definitions (numpy and scipy's
RegularGridInterpolator are their only dependencies) on seeded inputs. It
reads the reference checkout and is run by hand; the tests only read the .npz
it writes.

    python tests/golden/make_downsampling_golden.py /path/to/nlsolvers-datagen
"""
import ast
import os
import sys

import numpy as np
from scipy.interpolate import RegularGridInterpolator

NAMES = ["downsample_interpolation", "downsample_interpolation_3d"]


def load_functions(ref_root):
    rel = "scripts/downsampling.py"
    tree = ast.parse(open(os.path.join(ref_root, rel)).read())
    defs = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in NAMES]
    assert sorted(d.name for d in defs) == sorted(NAMES)
    ns = {"np": np, "RegularGridInterpolator": RegularGridInterpolator}
    exec(compile(ast.Module(body=defs, type_ignores=[]), rel, "exec"), ns)
    return ns


# (frames, source shape, target shape, domain half-widths, complex)
CASES_2D = [
    (2, (48, 48), (24, 24), (10.0, 10.0), False),
    (2, (37, 29), (17, 23), (8.0, 5.0), False),
    (1, (21, 21), (21, 21), (6.0, 6.0), False),   # same shape: the identity
    (1, (30, 26), (19, 14), (10.0, 7.0), True),
    (1, (16, 16), (29, 29), (5.0, 5.0), False),   # upsampling
]
CASES_3D = [
    (1, (16, 14, 12), (8, 7, 6), (10.0, 9.0, 8.0), False),
    (1, (13, 13, 13), (9, 5, 11), (6.0, 6.0, 6.0), True),
]


def field(rng, shape, cplx):
    axes = [np.linspace(-1, 1, n) for n in shape]
    grids = np.meshgrid(*axes, indexing="ij")
    f = np.exp(-sum((g - c) ** 2 for g, c in zip(grids, rng.uniform(-0.5, 0.5, len(shape)))) / 0.3)
    f = f + 0.1 * rng.standard_normal(shape)
    if cplx:
        f = f * np.exp(1j * rng.uniform(0, 2 * np.pi)) + 0.05j * rng.standard_normal(shape)
    return f


def main(ref_root):
    F = load_functions(ref_root)
    rng = np.random.default_rng(77)
    out = {}
    for i, (nf, shp, tgt, L, cplx) in enumerate(CASES_2D):
        u = np.stack([field(rng, shp, cplx) for _ in range(nf)])
        d = F["downsample_interpolation"](u, tgt, L[0], L[1])
        out[f"d2_{i}_in"], out[f"d2_{i}_out"] = u, d
        out[f"d2_{i}_L"] = np.array(L)
    for i, (nf, shp, tgt, L, cplx) in enumerate(CASES_3D):
        u = np.stack([field(rng, shp, cplx) for _ in range(nf)])
        d = F["downsample_interpolation_3d"](u, tgt, L[0], L[1], L[2])
        out[f"d3_{i}_in"], out[f"d3_{i}_out"] = u, d
        out[f"d3_{i}_L"] = np.array(L)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "downsampling.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, sorted(out))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NLS_REFERENCE_DIR", "")
    if not ref:
        sys.exit("usage: %s REFERENCE_CHECKOUT (or set NLS_REFERENCE_DIR)" % sys.argv[0])
    main(ref)
