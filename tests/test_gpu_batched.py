"""Blocks of right-hand sides (prism_solve_batched*, prism_apply_batched_device)
through the C ABI: every column against the single-vector path of the same
handle, which is itself parity-tested against the oracle and the reference.
Tolerances: applies 1e-12 relative (the block sweep sums a row's entries in
another order), solves: iteration counts within 1 and solutions within 1e-10
relative when the counts agree."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


PRECONDS = [(P.PRECOND_IC, P.PRISM_FP32), (P.PRECOND_IC, P.PRISM_FP64), (P.PRECOND_ILDLT, P.PRISM_FP64),
            (P.PRECOND_ILUT, P.PRISM_FP32)]


@pytest.mark.parametrize("kind,prec", PRECONDS)
@pytest.mark.parametrize("k", [1, 7, 64])
def test_block_apply_matches_single_apply(kind, prec, k):
    A = P.CSRMatrix.laplacian(24, 20, 12)
    S = P.DeviceSystem(A)
    S.set_precond(kind, tol=1e-3, precision=prec)
    V = np.random.default_rng(k).standard_normal((k, A.n))
    out = S.apply_batched(V)
    for c in range(k):
        assert rel_err(out[c], S.apply(V[c])) < 1e-12, c


def test_block_apply_vs_oracle():
    A = P.CSRMatrix.laplacian(32, 32, 8)
    F = P.HostFactor(A, P.PRECOND_IC, tol=1e-3, precision=P.PRISM_FP32)
    S = P.DeviceSystem(A)
    S.attach(F)
    rp, ci, v, _ = F.arrays(0)
    O = orc.Precond(1, A.n, (rp, ci, v))
    V = np.random.default_rng(3).standard_normal((16, A.n))
    out = S.apply_batched(V)
    for c in range(16):
        assert rel_err(out[c], O.apply(V[c])) < 1e-12


@pytest.mark.parametrize("kind,prec", [(P.PRECOND_IC, P.PRISM_FP32), (P.PRECOND_ILDLT, P.PRISM_FP64),
                                       (P.PRECOND_NONE, P.PRISM_FP64)])
def test_block_fcg_matches_single_solves(kind, prec):
    A = P.CSRMatrix.laplacian(48, 40, 1)
    S = P.DeviceSystem(A)
    S.set_precond(kind, tol=1e-3, precision=prec)
    k = 12
    rng = np.random.default_rng(5)
    B = rng.standard_normal((k, A.n))
    B[3] *= 1e-6          # columns converge at different iterations
    B[7] = rng.uniform(-1, 1, A.n)
    X, st = S.solve_batched(B, tol=1e-10, max_iter=2000)
    for c in range(k):
        x1, s1 = S.solve(B[c], tol=1e-10, max_iter=2000)
        assert st[c].converged and abs(st[c].num_iter - s1.num_iter) <= 1, (c, st[c].num_iter, s1.num_iter)
        if st[c].num_iter == s1.num_iter:
            assert rel_err(X[c], x1) < 1e-10, c
        assert st[c].true_rel_residual < 1.5e-10


def test_block_fcg_device_pointers_and_guess():
    import torch
    A = P.CSRMatrix.laplacian(64, 64, 1)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3, precision=P.PRISM_FP32)
    B = torch.from_numpy(np.random.default_rng(9).standard_normal((64, A.n))).cuda()
    X0 = torch.full_like(B, 0.5)
    X, st = S.solve_batched(B, X0, tol=1e-9)
    assert all(s.converged for s in st)
    x1, s1 = S.solve(B[17].cpu().numpy(), np.full(A.n, 0.5), tol=1e-9)
    assert abs(st[17].num_iter - s1.num_iter) <= 1
    if st[17].num_iter == s1.num_iter:
        assert rel_err(X[17].cpu().numpy(), x1) < 1e-10


def test_block_rejects_bad_sizes_and_solver():
    A = P.CSRMatrix.laplacian(8, 8, 1)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3)
    with pytest.raises(P.PrismError):
        S.solve_batched(np.ones((65, A.n)))
    with pytest.raises(P.PrismError):
        S.solve_batched(np.ones((2, A.n)), solver=P.SOLVER_FGMRES)
