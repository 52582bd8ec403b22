"""The oracle's fixed-pattern refactorisation (orc_refactor: the reference's
IncompleteCholesky / IncompleteLDLT setup with the drop test replaced by the
given pattern) against the host factorisation, which is itself bit-exact with
the compiled reference: with the matrix the factor was built from, the
refactorisation must return the same values to the last bit."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P
from oracle import oracle as orc


@pytest.mark.parametrize("kind,tol", [(P.PRECOND_IC, 1e-3), (P.PRECOND_IC, 0.0), (P.PRECOND_ILDLT, 1e-3)])
@pytest.mark.parametrize("precision", [P.PRISM_FP64, P.PRISM_FP32])
def test_refactor_on_own_pattern_reproduces_host_factor(kind, tol, precision):
    A = P.CSRMatrix.laplacian(11, 9, 7)
    F = P.HostFactor(A, kind, tol=tol, precision=precision)
    rp, ci, v, d = F.arrays(0)
    rc, lv, D = orc.refactor(kind, A.rowptr, A.col, A.val, rp, ci, single=precision == P.PRISM_FP32)
    assert rc == 0
    assert np.array_equal(lv, v)
    if kind == P.PRECOND_ILDLT:
        assert np.array_equal(D, d)


def test_refactor_reports_a_non_positive_pivot():
    A = P.CSRMatrix.laplacian(6, 6, 1)
    F = P.HostFactor(A, P.PRECOND_IC, tol=1e-3)
    rp, ci, _, _ = F.arrays(0)
    rc, _, _ = orc.refactor(P.PRECOND_IC, A.rowptr, A.col, -A.val, rp, ci)
    assert rc == 4
