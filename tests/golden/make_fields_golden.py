"""Generate tests/golden/fields.npz from the reference's own coefficient-field
generators: generate_m_fields (scripts/m_fields_2d.py:147-238) and
generate_c_fields (scripts/c_fields_2d.py:169-248), with the functions they
call. The modules import matplotlib at the top (absent here), so this script
parses the two files and executes only their field definitions (numpy and
scipy.ndimage / scipy.spatial are their dependencies), on seeded calls: every
m kind (with a c field for the kinds that need one) and every c kind, a few
fields each so that the random choices inside each kind vary, plus the default
calls that mix all kinds. It reads the reference checkout and is run by hand;
the tests only read the .npz it writes.

    python tests/golden/make_fields_golden.py /path/to/nlsolvers-datagen
"""
import ast
import os
import sys

import numpy as np
from scipy.ndimage import gaussian_filter, laplace
from scipy.signal import convolve2d
from scipy.spatial.distance import cdist

M_KINDS = ['constant', 'piecewise', 'gradient', 'phase', 'topological', 'defects', 'quasiperiodic', 'multiscale']
C_KINDS = ['periodic_structure', 'piecewise_constant', 'sign_changing_mass', 'layered', 'waveguide',
           'quasiperiodic', 'turbulent', 'constant']


def load(ref_root, rel):
    tree = ast.parse(open(os.path.join(ref_root, rel)).read())
    defs = [nd for nd in tree.body if isinstance(nd, ast.FunctionDef) and not nd.name.startswith('visualize')]
    ns = {"np": np, "gaussian_filter": gaussian_filter, "laplace": laplace, "cdist": cdist,
          "convolve2d": convolve2d}
    exec(compile(ast.Module(body=defs, type_ignores=[]), rel, "exec"), ns)
    return ns


def main(ref_root):
    Mf = load(ref_root, "scripts/m_fields_2d.py")
    Cf = load(ref_root, "scripts/c_fields_2d.py")
    out = {}
    n, L = 48, 5.0
    # a smooth c field for the m kinds built from one
    c_in = Cf["periodic_structure"](n, L, amplitude=0.4, frequency=2)
    out["c_in"] = c_in
    for i, kind in enumerate(M_KINDS):
        np.random.seed(100 + i)
        fields, _ = Mf["generate_m_fields"](n, L, c_field=c_in, num_fields=3, field_types=[kind] * 3)
        out[f"m_{kind}"] = np.stack(fields)
    for i, kind in enumerate(C_KINDS):
        fields, _ = Cf["generate_c_fields"](n, L, num_fields=3, field_types=[kind], seed=200 + i)
        out[f"c_{kind}"] = np.stack(fields)
    # the default calls: every m kind in order, and c kinds drawn at random
    np.random.seed(7)
    out["m_default"] = np.stack(Mf["generate_m_fields"](40, 6.0, c_field=c_in[:40, :40])[0])
    out["c_default"] = np.stack(Cf["generate_c_fields"](40, 6.0, num_fields=7, seed=8)[0])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fields.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, sorted(out))


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NLS_REFERENCE_DIR", "")
    if not ref:
        sys.exit("usage: %s REFERENCE_CHECKOUT (or set NLS_REFERENCE_DIR)" % sys.argv[0])
    main(ref)
