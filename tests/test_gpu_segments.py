"""Batches of independent systems solved together (prism_solve_segments*):
uneven 2D Poisson systems assembled on the diagonal of one CSR, one
preconditioner over the whole batch, each system on its own CG scalars --
checked against each system solved alone on the device and by the oracle
(iteration counts within +-1, solutions within 1e-10 at equal counts)."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


SIDES = [8, 23, 40, 17, 31, 12, 36]


def batch(sides, seed=5):
    blocks = [P.CSRMatrix.laplacian(s, s, 1) for s in sides]
    A, seg = P.CSRMatrix.block_diagonal(blocks)
    b = np.random.default_rng(seed).standard_normal(A.n)
    return blocks, A, seg, b


@pytest.mark.parametrize("kind,prec", [(P.PRECOND_IC, P.PRISM_FP64), (P.PRECOND_ILDLT, P.PRISM_FP32)])
def test_segments_match_single_solves(kind, prec):
    blocks, A, seg, b = batch(SIDES)
    S = P.DeviceSystem(A)
    S.set_precond(kind, tol=1e-3, precision=prec)
    x, stats = S.solve_segments(seg, b, tol=1e-10, max_iter=2000)
    for s, B in enumerate(blocks):
        lo, hi = seg[s], seg[s + 1]
        Si = P.DeviceSystem(B)
        Si.set_precond(kind, tol=1e-3, precision=prec)
        xi, sti = Si.solve(b[lo:hi], tol=1e-10, max_iter=2000)
        assert stats[s].converged and abs(stats[s].num_iter - sti.num_iter) <= 1, (s, stats[s].num_iter, sti.num_iter)
        if stats[s].num_iter == sti.num_iter:
            assert rel_err(x[lo:hi], xi) < 1e-10, s
        assert stats[s].true_rel_residual < 1.5e-10


def test_segments_against_oracle():
    blocks, A, seg, b = batch(SIDES, seed=9)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3)
    x, stats = S.solve_segments(seg, b, tol=1e-8, max_iter=1000)
    for s, B in enumerate(blocks):
        lo, hi = seg[s], seg[s + 1]
        F = P.HostFactor(B, P.PRECOND_IC, tol=1e-3)
        rp, ci, v, _ = F.arrays(0)
        xo, ito, _, _ = orc.cg(B.rowptr, B.col, B.val, b[lo:hi], orc.Precond(1, B.n, (rp, ci, v)), tol=1e-8,
                               maxit=1000)
        assert abs(stats[s].num_iter - ito) <= 1
        if stats[s].num_iter == ito:
            assert rel_err(x[lo:hi], xo) < 1e-10


def test_segments_device_path_repeatable_and_zero_rhs():
    import torch
    blocks, A, seg, b = batch([20, 9, 27])
    b[seg[1]:seg[2]] = 0.0  # the middle system has b = 0
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3)
    bd = torch.tensor(b, device="cuda")
    x1, st1 = S.solve_segments(seg, bd, tol=1e-10)
    x2, st2 = S.solve_segments(seg, bd, tol=1e-10)
    torch.cuda.synchronize()
    assert torch.equal(x1, x2)
    assert st1[1].converged and st1[1].num_iter == 1
    assert not torch.any(x1[seg[1]:seg[2]] != 0)
    xh, _ = S.solve_segments(seg, b, tol=1e-10)
    assert rel_err(xh, x1.cpu().numpy()) == 0.0


def test_segments_reject_coupled_rows():
    A = P.CSRMatrix.laplacian(10, 10, 1)
    S = P.DeviceSystem(A)
    with pytest.raises(P.PrismError) as e:
        S.solve_segments(np.array([0, 50, 100], np.uint32), np.ones(A.n))
    assert e.value.status == 1
