"""The oracle's restatement of the reference's linear-interpolation
downsampling (scripts/downsampling.py:68-103, :215-257) against the golden
vectors made from the reference's own functions
(tests/golden/make_downsampling_golden.py): equal bitwise."""
import os

import numpy as np
import pytest

from oracle import downsample as D

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "downsampling.npz")


def _cases():
    g = np.load(GOLDEN)
    return [(k[:-3], g[k], g[k[:-3] + "_out"], g[k[:-3] + "_L"]) for k in sorted(g) if k.endswith("_in")]


@pytest.mark.parametrize("name,u,ref,L", _cases(), ids=[c[0] for c in _cases()])
def test_oracle_downsampling_equals_reference(name, u, ref, L):
    out = D.downsample_interpolation(u, ref.shape[1:], L)
    assert out.dtype == ref.dtype and out.shape == ref.shape
    assert np.array_equal(out, ref)


def test_linspace_matches_numpy():
    for L, n in [(10.0, 300), (15.0, 128), (7.3, 33), (1.0, 2)]:
        assert np.array_equal(D.linspace(L, n), np.linspace(-L, L, n))
