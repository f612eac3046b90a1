"""Generate tests/golden/fft_downsampling.npz from the reference's own spectral
downsampling.

The reference defines downsample_fft (scripts/downsampling.py:10-35, 2-D) and
downsample_fft_3d (:147-178, 3-D): the orthonormal DFT of every frame, the
centred crop of the fftshift-ed spectrum to the target shape, and the inverse
DFT (real inputs keep the real part). Its 3-D NLSE launcher applies the 3-D
one to the snapshots (scripts/complex_launcher_3d.py:185-187). The module
imports matplotlib at the top (absent here), so this script parses the file
and executes only those two function definitions, with numpy and torch (on
the CPU) as their dependencies, on seeded inputs. It reads the reference
checkout and is run by hand; the tests only read the .npz it writes.

    python tests/golden/make_fft_downsampling_golden.py /path/to/nlsolvers-datagen
"""
import ast
import os
import sys

import numpy as np
import torch

NAMES = ["downsample_fft", "downsample_fft_3d"]


def load_functions(ref_root):
    rel = "scripts/downsampling.py"
    tree = ast.parse(open(os.path.join(ref_root, rel)).read())
    defs = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in NAMES]
    assert sorted(d.name for d in defs) == sorted(NAMES)
    ns = {"np": np, "torch": torch}
    exec(compile(ast.Module(body=defs, type_ignores=[]), rel, "exec"), ns)
    return ns


# (frames, source shape, target shape, complex): even and odd extents on both
# sides of the crop, an axis left whole, and the snapshot sizes of the
# 128^2 -> 48^2 case
CASES_2D = [
    (2, (40, 40), (16, 16), False),
    (2, (37, 41), (17, 20), False),
    (1, (33, 30), (33, 29), False),
    (2, (40, 36), (15, 18), True),
    (1, (29, 31), (10, 9), True),
    (1, (128, 128), (48, 48), True),
]
CASES_3D = [
    (2, (20, 18, 16), (8, 9, 10), False),
    (1, (17, 16, 15), (8, 8, 7), True),
    (1, (24, 24, 24), (12, 12, 12), True),
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
    rng = np.random.default_rng(78)
    out = {}
    for i, (nf, shp, tgt, cplx) in enumerate(CASES_2D):
        u = np.stack([field(rng, shp, cplx) for _ in range(nf)])
        out[f"f2_{i}_in"], out[f"f2_{i}_out"] = u, F["downsample_fft"](u, tgt)
    for i, (nf, shp, tgt, cplx) in enumerate(CASES_3D):
        u = np.stack([field(rng, shp, cplx) for _ in range(nf)])
        out[f"f3_{i}_in"], out[f"f3_{i}_out"] = u, F["downsample_fft_3d"](u, tgt)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fft_downsampling.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, sorted(out))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NLS_REFERENCE_DIR", "")
    if not ref:
        sys.exit("usage: %s REFERENCE_CHECKOUT (or set NLS_REFERENCE_DIR)" % sys.argv[0])
    main(ref)
