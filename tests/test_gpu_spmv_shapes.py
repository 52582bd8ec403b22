"""The SpMV kernel's shapes (lanes per row, rows per pass), which prism_create
chooses among by timing: every shape computes A x as the oracle's CSR product
(CSRMatrix::MatPVec, include/MatrixClass/CSRMatrix.h:360-395) to rounding, on
short stencil rows and on long rows, and a solve converges with each."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

SHAPES = [(1, 2), (1, 4), (2, 2), (4, 1), (8, 1), (16, 1)]


def long_rows(n=3000, per=70, seed=3):
    """Symmetric, diagonally dominant, about `per` entries per row, rows of uneven length."""
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    M = sp.random(n, n, density=per / (2 * n), random_state=rng, format="csr")
    M = M + M.T
    M = M + sp.diags(np.asarray(abs(M).sum(axis=1)).ravel() + 1.0)
    M = M.tocsr()
    M.sort_indices()
    return P.CSRMatrix(M.indptr, M.indices, M.data)


@pytest.mark.parametrize("shape", range(len(SHAPES)))
@pytest.mark.parametrize("which", ["poisson", "long"])
def test_every_shape_matches_the_oracle(monkeypatch, shape, which):
    monkeypatch.setenv("PRISM_SPMV_SHAPE", str(shape))
    A = P.CSRMatrix.laplacian(40, 30, 20) if which == "poisson" else long_rows()
    S = P.DeviceSystem(A)
    assert S.spmv_shape() == SHAPES[shape]
    x = np.random.default_rng(shape).standard_normal(A.n)
    y = S.spmv(x)
    ref = orc.spmv(A.rowptr, A.col, A.val, x)
    assert np.abs(y - ref).max() <= 1e-14 * np.abs(ref).max() * 8
    b = np.random.default_rng(7).standard_normal(A.n)
    _, st = S.solve(b, tol=1e-10, max_iter=2000)
    assert st.converged and st.true_rel_residual < 1e-9


def test_tuned_shape_is_one_of_the_table():
    for A in (P.CSRMatrix.laplacian(64, 64, 64), long_rows(20000, 120)):
        S = P.DeviceSystem(A)
        assert S.spmv_shape() in SHAPES
