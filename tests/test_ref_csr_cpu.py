"""The CSR arrays that carry the operator to the reference's compiled device
code (oracle/ref_kg.py) equal the oracle's matrix-free operator: A x from the
CSR matches apply_operator on random fields, 2-D and 3-D, both signs."""
import numpy as np
import pytest
import scipy.sparse as sp

import nlsb200 as nl
from nlsb200 import workloads as W
from oracle import oracle as O
from oracle import ref_kg


@pytest.mark.parametrize("dim,n", [(2, 24), (2, 37), (3, 9)])
@pytest.mark.parametrize("sign", [-1.0, 1.0])
def test_csr_matches_operator(dim, n, sign):
    spec, *_ = W.kg_case(n, 8.0, T=0.1, nt=10, ns=1, k=10, seed=3, dim=dim, precision=nl.FP64)
    ip, ix, vals = ref_kg.csr(spec, sign)
    A = sp.csr_matrix((vals, ix, ip), shape=(spec.n, spec.n))
    x = np.random.default_rng(n).standard_normal(spec.shape)
    dx = 2 * spec.Lx / (spec.nx - 1)
    y = O.apply_operator(x, np.ones(spec.shape), dim, 1.0 / (dx * dx), sign)
    assert np.abs(A @ x.ravel() - y.ravel()).max() <= 1e-12 * np.abs(y).max()
    assert (abs(A - A.T) > 0).nnz == 0
