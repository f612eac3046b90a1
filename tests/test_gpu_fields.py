"""Coefficient fields generated on the GPU (nlsb200.fields, nls_field2d) against
the reference's own generators (tests/golden/fields.npz, made by
tests/golden/make_fields_golden.py from scripts/m_fields_2d.py and
scripts/c_fields_2d.py): every m kind and c kind, a few fields each, and the
default mixed calls, with the same seeds. Tolerance 1e-12 relative per call
(FP64; the device's convolutions and reductions sum in their own order and
its tanh / exp / sin are CUDA's, so the agreement is not bitwise)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "fields.npz")
M_KINDS = ['constant', 'piecewise', 'gradient', 'phase', 'topological', 'defects', 'quasiperiodic', 'multiscale']
C_KINDS = ['periodic_structure', 'piecewise_constant', 'sign_changing_mass', 'layered', 'waveguide',
           'quasiperiodic', 'turbulent', 'constant']
TOL = 1e-12


def _close(got, want):
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape
    err = np.linalg.norm((got - want).ravel()) / np.linalg.norm(want.ravel())
    assert err < TOL, err


@pytest.mark.parametrize("kind", M_KINDS)
def test_m_fields_on_device(kind):
    from nlsb200 import fields as F
    g = np.load(GOLDEN)
    np.random.seed(100 + M_KINDS.index(kind))
    out, _ = F.generate_m_fields(48, 5.0, c_field=g["c_in"], num_fields=3, field_types=[kind] * 3)
    _close(np.stack(out), g[f"m_{kind}"])


@pytest.mark.parametrize("kind", C_KINDS)
def test_c_fields_on_device(kind):
    from nlsb200 import fields as F
    g = np.load(GOLDEN)
    out, _ = F.generate_c_fields(48, 5.0, num_fields=3, field_types=[kind], seed=200 + C_KINDS.index(kind))
    _close(np.stack(out), g[f"c_{kind}"])


def test_default_mixed_calls_on_device():
    from nlsb200 import fields as F
    g = np.load(GOLDEN)
    np.random.seed(7)
    _close(np.stack(F.generate_m_fields(40, 6.0, c_field=g["c_in"][:40, :40])[0]), g["m_default"])
    _close(np.stack(F.generate_c_fields(40, 6.0, num_fields=7, seed=8)[0]), g["c_default"])
