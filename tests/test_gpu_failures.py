"""Failures injected on the host, never on the device: a NaN in the
right-hand side, NaN values in A's factor, a NaN in the middle of a batch.

The library must answer each with a status (PRISM_ERR_NONFINITE = 7 for a NaN
met in a Krylov scalar, PRISM_ERR_NOT_SPD / ZERO_PIVOT when the host
factorisation sees it first) and never with PRISM_ERR_TIMEOUT (6): the
sweeps' readiness encoding is a signalling-NaN bit pattern no arithmetic
result takes, so a NaN result must count as finished, not as pending.  After
each failure the same handle must still solve a valid system."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P

pytestmark = pytest.mark.gpu

PRECISIONS = [P.PRISM_FP64, P.PRISM_FP32, P.PRISM_FP32_APPLY]


def _still_solves(S, A, rng):
    b = rng.standard_normal(A.n)
    x, st = S.solve(b, tol=1e-10, max_iter=1000)
    assert st.converged and st.true_rel_residual <= 1e-10


@pytest.mark.parametrize("precision", PRECISIONS)
def test_nan_rhs_gives_nonfinite_not_timeout(precision):
    rng = np.random.default_rng(1)
    A = P.CSRMatrix.laplacian(24, 24, 24)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3, precision=precision)
    b = rng.standard_normal(A.n)
    b[A.n // 3] = np.nan
    with pytest.raises(P.PrismError) as e:
        S.solve(b, tol=1e-10, max_iter=200)
    assert e.value.status == 7, str(e.value)
    _still_solves(S, A, rng)


def test_nan_rhs_through_amsed_and_fgmres():
    rng = np.random.default_rng(2)
    A = P.CSRMatrix.laplacian(24, 24, 24)
    S = P.DeviceSystem(A)
    S.set_amsed(precision=P.PRISM_FP32_APPLY, levels=3, lanczos_steps=16, low_rank=8, lowrank_type=0, reorder=0)
    b = rng.standard_normal(A.n)
    b[7] = np.inf
    for solver, restart in ((P.SOLVER_FCG, 0), (P.SOLVER_FGMRES, 30)):
        with pytest.raises(P.PrismError) as e:
            S.solve(b, solver=solver, tol=1e-10, max_iter=200, restart=restart)
        assert e.value.status == 7, str(e.value)
    _still_solves(S, A, rng)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_nan_matrix_values_are_reported_not_waited_on(precision):
    """A NaN among A's values: the refactorised preconditioner (or the solve it
    feeds) reports a status; a sweep never waits on a NaN result."""
    rng = np.random.default_rng(3)
    A = P.CSRMatrix.laplacian(20, 20, 20)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3, precision=precision)
    bad = A.val.copy()
    bad[len(bad) // 2] = np.nan
    S.update_values(bad)
    with pytest.raises(P.PrismError) as e:
        S.set_precond(P.PRECOND_IC, tol=1e-3, precision=precision)
        S.solve(rng.standard_normal(A.n), tol=1e-10, max_iter=200)
    assert e.value.status in (3, 4, 7), str(e.value)
    S.update_values(A.val)
    S.set_precond(P.PRECOND_IC, tol=1e-3, precision=precision)
    _still_solves(S, A, rng)


def test_nan_in_one_block_column_stops_with_status():
    rng = np.random.default_rng(4)
    A = P.CSRMatrix.laplacian(32, 32, 1)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3)
    B = rng.standard_normal((4, A.n))
    B[2, 5] = np.nan
    with pytest.raises(P.PrismError) as e:
        S.solve_batched(B, tol=1e-10, max_iter=200)
    assert e.value.status == 7, str(e.value)
    _still_solves(S, A, rng)
