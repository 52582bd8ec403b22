"""Host model problems: the upwind convection-diffusion operator and
block-diagonal assembly of a batch of systems (no GPU)."""
from __future__ import annotations

import numpy as np

import prispack_b200 as P


def test_convection_diffusion_pattern_and_limits():
    A = P.CSRMatrix.convection_diffusion(7, 6, 5, 50.0, 25.0, 12.5)
    L = P.CSRMatrix.laplacian(7, 6, 5)
    assert np.array_equal(A.rowptr, L.rowptr) and np.array_equal(A.col, L.col)
    # zero velocity is the 7-point Laplacian of generateLaplacianCSR
    A0 = P.CSRMatrix.convection_diffusion(7, 6, 5, 0.0, 0.0, 0.0)
    assert np.array_equal(A0.val, L.val)
    # M-matrix: positive diagonal, non-positive off-diagonals, weak row diagonal dominance
    M = A.to_scipy().toarray()
    assert np.all(np.diag(M) > 0) and np.all(M - np.diag(np.diag(M)) <= 0)
    assert np.all(M.sum(axis=1) >= -1e-12)
    # upwind: for v_x > 0 the upstream (x - 1) neighbour carries 1 + h v_x, the downstream one 1
    h = 1.0 / 8
    i = 2 + 7 * (2 + 6 * 2)
    assert np.isclose(M[i, i - 1], -(1.0 + h * 50.0)) and np.isclose(M[i, i + 1], -1.0)
    assert not np.allclose(M, M.T)


def test_block_diagonal_assembly():
    blocks = [P.CSRMatrix.laplacian(s, s, 1) for s in (3, 5, 4)]
    A, seg = P.CSRMatrix.block_diagonal(blocks)
    assert list(seg) == [0, 9, 34, 50] and A.nnz == sum(B.nnz for B in blocks)
    D = A.to_scipy().toarray()
    for s, B in enumerate(blocks):
        lo, hi = seg[s], seg[s + 1]
        assert np.array_equal(D[lo:hi, lo:hi], B.to_scipy().toarray())
        assert not D[lo:hi, :lo].any() and not D[lo:hi, hi:].any()
