"""Generate tests/golden/diagnostics.npz from the reference's own Python
diagnostics.

The reference computes energy and mass post hoc in
scripts/compare_utils_real_2d.py:112-131 (compute_gradient_sq_norm,
compute_mass, compute_hamiltonian_kge_u_cubed) and
scripts/compare_utils_complex_2d.py:134-151 (compute_gradient_sq_norm_complex_std,
compute_mass_nlse, compute_hamiltonian_nlse_std). Those modules import
matplotlib and other packages at the top, so this script parses each file and
executes only those function definitions (numpy is their only dependency) on
seeded inputs. It reads the reference checkout and is run by hand; the tests
only read the .npz it writes.

    python tests/golden/make_diagnostics_golden.py /path/to/nlsolvers-datagen
"""
import ast
import os
import sys

import numpy as np

FUNCS = {
    "scripts/compare_utils_real_2d.py": ["compute_gradient_sq_norm", "compute_mass",
                                         "compute_hamiltonian_kge_u_cubed"],
    "scripts/compare_utils_complex_2d.py": ["compute_gradient_sq_norm_complex_std",
                                            "compute_mass_nlse", "compute_hamiltonian_nlse_std"],
}


def load_functions(ref_root):
    ns = {"np": np}
    for rel, names in FUNCS.items():
        tree = ast.parse(open(os.path.join(ref_root, rel)).read())
        defs = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
        assert sorted(d.name for d in defs) == sorted(names), rel
        exec(compile(ast.Module(body=defs, type_ignores=[]), rel, "exec"), ns)
    return ns


def smooth(rng, ny, nx, L):
    x = np.linspace(-L, L, nx)
    y = np.linspace(-L, L, ny)
    X, Y = np.meshgrid(x, y)
    f = np.zeros((ny, nx))
    for _ in range(3):
        a, w = rng.uniform(0.5, 2.0), rng.uniform(0.5, 2.0)
        cx, cy = rng.uniform(-0.6 * L, 0.6 * L, 2)
        f += a * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * w * w))
    return f


def main(ref_root):
    F = load_functions(ref_root)
    rng = np.random.default_rng(2024)
    out = {}
    # KG cases: (nx, ny, Lx, Ly, with c)
    for i, (nx, ny, Lx, Ly, with_c) in enumerate([(24, 24, 5.0, 5.0, True), (31, 20, 6.0, 4.0, False)]):
        u = smooth(rng, ny, nx, Lx) + 0.05 * rng.standard_normal((ny, nx))
        v = 0.3 * rng.standard_normal((ny, nx))
        m = 1.0 + 0.2 * rng.standard_normal((ny, nx))
        c = 1.0 + 0.3 * rng.random((ny, nx)) if with_c else np.ones((ny, nx))
        dx, dy = 2 * Lx / (nx - 1), 2 * Ly / (ny - 1)  # compare_utils_real_2d.py:301-302
        e_ut, e_grad, e_pot = F["compute_hamiltonian_kge_u_cubed"](u, v, dx, dy, m, c)
        mass = F["compute_mass"](u, dx, dy)
        out[f"kg{i}_geom"] = np.array([nx, ny, Lx, Ly])
        out[f"kg{i}_u"], out[f"kg{i}_v"], out[f"kg{i}_m"], out[f"kg{i}_c"] = u, v, m, c
        out[f"kg{i}_diag"] = np.array([e_ut, e_grad, e_pot, mass])
    # NLSE cases
    for i, (nx, ny, Lx, Ly) in enumerate([(26, 26, 5.0, 5.0), (19, 33, 3.0, 7.0)]):
        amp = smooth(rng, ny, nx, Lx)
        ph = rng.uniform(0, 2 * np.pi) + 0.4 * np.linspace(-Lx, Lx, nx)[None, :]
        u = amp * np.exp(1j * ph) + 0.02 * (rng.standard_normal((ny, nx)) + 1j * rng.standard_normal((ny, nx)))
        dx, dy = 2 * Lx / (nx - 1), 2 * Ly / (ny - 1)  # compare_utils_complex_2d.py:311-312
        e_grad, e_pot = F["compute_hamiltonian_nlse_std"](u, dx, dy)
        mass = F["compute_mass_nlse"](u, dx, dy)
        out[f"nlse{i}_geom"] = np.array([nx, ny, Lx, Ly])
        out[f"nlse{i}_u"] = u
        out[f"nlse{i}_diag"] = np.array([mass, e_grad, e_pot, 0.0])
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "diagnostics.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, {k: v.tolist() for k, v in out.items() if k.endswith("diag")})


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NLS_REFERENCE_DIR", "")
    if not ref:
        sys.exit("usage: %s REFERENCE_CHECKOUT (or set NLS_REFERENCE_DIR)" % sys.argv[0])
    main(ref)
