"""Single-precision apply (PRISM_FP32_APPLY): float factor values and float
arithmetic inside the streamed triangular sweeps, double everywhere else.

The reference has no such mode (its float instantiation, PRISM_FP32 here,
computes in double), so the checks are: the apply agrees with the PRISM_FP32
apply to single-precision accuracy (relative 2-norm difference <= 1e-5), the
sweeps run on the streamed kernel, and the flexible outer solvers still reach
a 1e-10 true relative residual with about as many iterations."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P

pytestmark = pytest.mark.gpu

APPLY_RTOL = 1e-5


def rel2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _pair(A, setup):
    """Two systems on A whose preconditioners differ only in precision."""
    S32, S1 = P.DeviceSystem(A), P.DeviceSystem(A)
    setup(S32, P.PRISM_FP32)
    setup(S1, P.PRISM_FP32_APPLY)
    return S32, S1


@pytest.mark.parametrize("kind", [P.PRECOND_IC, P.PRECOND_ILDLT])
def test_symmetric_apply_matches_fp32_storage(kind):
    A = P.CSRMatrix.laplacian(24, 24, 24)
    S32, S1 = _pair(A, lambda S, p: S.set_precond(kind, tol=1e-3, precision=p))
    for sw in (0, 1):
        assert S1.sweep_info(sw)["kernel"] == "stream"
    v = np.random.default_rng(3).standard_normal(A.n)
    ref, got = S32.apply(v), S1.apply(v)
    assert np.isfinite(got).all()
    assert rel2(got, ref) < APPLY_RTOL


def test_ilut_apply_and_fgmres_nonsymmetric():
    A = P.CSRMatrix.convection_diffusion(20, 20, 20, 10.0, 5.0, 2.5)
    S32, S1 = _pair(A, lambda S, p: S.set_precond(P.PRECOND_ILUT, tol=1e-3, lfill=20, precision=p))
    v = np.random.default_rng(4).standard_normal(A.n)
    assert rel2(S1.apply(v), S32.apply(v)) < APPLY_RTOL
    b = np.random.default_rng(5).standard_normal(A.n)
    _, st32 = S32.solve(b, solver=P.SOLVER_FGMRES, tol=1e-10, max_iter=500, restart=50)
    x, st = S1.solve(b, solver=P.SOLVER_FGMRES, tol=1e-10, max_iter=500, restart=50)
    # FGMRES stops on its Givens residual estimate (as the reference's does); the true
    # residual at exit stays within a small factor of the tolerance
    assert st.converged and st.true_rel_residual <= 1e-9
    assert abs(st.num_iter - st32.num_iter) <= 3


def test_amsed_fcg_reaches_1e10():
    A = P.CSRMatrix.laplacian(32, 32, 32)
    opts = dict(levels=3, lanczos_steps=32, low_rank=16, lowrank_type=0, reorder=0)
    S32, S1 = _pair(A, lambda S, p: S.set_amsed(precision=p, **opts))
    v = np.random.default_rng(6).standard_normal(A.n)
    assert rel2(S1.apply(v), S32.apply(v)) < APPLY_RTOL
    b = np.random.default_rng(7).standard_normal(A.n)
    _, st32 = S32.solve(b, tol=1e-10, max_iter=500)
    x, st = S1.solve(b, tol=1e-10, max_iter=500)
    assert st.converged and st.true_rel_residual <= 1e-10
    assert abs(st.num_iter - st32.num_iter) <= 3
    r = b - A.to_scipy() @ x
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-10


def test_block_solve_falls_back_to_double_sweeps():
    """Block solves run level-order sweeps in double; the result matches the
    single-vector solves of the same preconditioner to the solve tolerance."""
    A = P.CSRMatrix.laplacian(16, 16, 16)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3, precision=P.PRISM_FP32_APPLY)
    B = np.random.default_rng(8).standard_normal((4, A.n))
    X, stats = S.solve_batched(B, tol=1e-10, max_iter=500)
    for c in range(4):
        assert stats[c].converged and stats[c].true_rel_residual <= 1e-10
        xc, _ = S.solve(B[c], tol=1e-12, max_iter=500)
        assert rel2(np.asarray(X[c]), xc) < 1e-7


def test_precision_out_of_range_rejected():
    A = P.CSRMatrix.laplacian(6, 6, 1)
    S = P.DeviceSystem(A)
    with pytest.raises(P.PrismError, match="precision"):
        S.set_precond(P.PRECOND_IC, precision=3)
