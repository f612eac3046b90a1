"""The coefficient-field drop-ins (nlsb200/fields.py: generate_m_fields,
generate_c_fields) on CPU: with the oracle's numpy evaluation of the device
call's parameter layouts (oracle/fields.py) in place of nls_field2d, the
product's draws (numpy's global generator, in the reference's order) and its
parameter packing reproduce the reference's own generators' outputs
(tests/golden/fields.npz, tests/golden/make_fields_golden.py) to 1e-12
relative, for every m and c kind and for the default mixed calls."""
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "fields.npz")
M_KINDS = ['constant', 'piecewise', 'gradient', 'phase', 'topological', 'defects', 'quasiperiodic', 'multiscale']
C_KINDS = ['periodic_structure', 'piecewise_constant', 'sign_changing_mass', 'layered', 'waveguide',
           'quasiperiodic', 'turbulent', 'constant']
TOL = 1e-12


@pytest.fixture
def F(monkeypatch):
    from nlsb200 import fields
    from oracle import fields as OF
    monkeypatch.setattr(fields, "field2d", OF.evaluate)
    return fields


def _close(got, want):
    got, want = np.asarray(got), np.asarray(want)
    assert got.shape == want.shape
    err = np.linalg.norm((got - want).ravel()) / np.linalg.norm(want.ravel())
    assert err < TOL, err


@pytest.mark.parametrize("kind", M_KINDS)
def test_m_fields_against_reference(F, kind):
    g = np.load(GOLDEN)
    i = M_KINDS.index(kind)
    np.random.seed(100 + i)
    fields, params = F.generate_m_fields(48, 5.0, c_field=g["c_in"], num_fields=3, field_types=[kind] * 3)
    _close(np.stack(fields), g[f"m_{kind}"])
    assert all(p["type"] == kind for p in params)


@pytest.mark.parametrize("kind", C_KINDS)
def test_c_fields_against_reference(F, kind):
    g = np.load(GOLDEN)
    i = C_KINDS.index(kind)
    fields, _ = F.generate_c_fields(48, 5.0, num_fields=3, field_types=[kind], seed=200 + i)
    _close(np.stack(fields), g[f"c_{kind}"])


def test_default_mixed_calls(F):
    g = np.load(GOLDEN)
    np.random.seed(7)
    _close(np.stack(F.generate_m_fields(40, 6.0, c_field=g["c_in"][:40, :40])[0]), g["m_default"])
    _close(np.stack(F.generate_c_fields(40, 6.0, num_fields=7, seed=8)[0]), g["c_default"])


def test_gaussian_weights_match_scipy():
    from scipy.ndimage import gaussian_filter1d
    from nlsb200.fields import gaussian_weights
    rng = np.random.default_rng(0)
    v = rng.standard_normal(200)
    for sigma in (1.0, 2.7, 13.3, 29.9):
        w = gaussian_weights(sigma)
        from scipy.ndimage import correlate1d
        assert np.array_equal(correlate1d(v, w, mode='reflect'), gaussian_filter1d(v, sigma))


def test_malformed_parameters_are_rejected():
    """nls_field2d checks each kind's parameter layout and input count before
    any device call (no GPU needed)."""
    from nlsb200 import fields
    from nlsb200._lib import NlsError
    with pytest.raises(NlsError):
        fields.field2d(fields.M_DEFECTS, 16, 1.0, [1.0, 3.0, 0.0])   # 3 defects announced, none given
    with pytest.raises(NlsError):
        fields.field2d(fields.M_GRADIENT, 16, 1.0, [1.0, 1.0, 0.1])  # needs the c field
    with pytest.raises(NlsError):
        fields.field2d(fields.M_MULTISCALE, 16, 1.0, [1.0, 1.0, 0.5, 2.0, 0.5, 0.5], [np.zeros((16, 16))])
    with pytest.raises(NlsError):
        fields.field2d(99, 16, 1.0, [])
