"""The AMSED / MSLR apply on a block of right-hand sides, and its low-rank
block products on the tensor cores.

The low-rank correction x2 += W (H o (W^T xc)) (AMSEDPrecondition.cpp:
1557-1574) of k columns is two matrix products.  With FP64 factor values they
run in FP64 and the block apply must equal the single-vector apply column by
column to rounding (1e-12 relative).  With FP32 factor values they run on the
tensor cores with BF16 operands and FP32 accumulation; the kernels are checked
against a numpy emulation of exactly that arithmetic, with a bound that allows
the one BF16 rounding of the intermediate T = H o (W^T X) to land on the other
side of a rounding boundary (a relative 2^-8 of one term), and the block apply
against the single-vector apply within the BF16 error of the low-rank term."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P

pytestmark = pytest.mark.gpu

BF16_EPS = 2.0 ** -8


def bf16(a):
    """float64 -> float32 -> BF16 (round to nearest even) -> float64, as the kernels round."""
    f = np.ascontiguousarray(a, np.float64).astype(np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


@pytest.mark.parametrize("nrem,rank,k", [(1000, 20, 64), (517, 37, 13), (64, 6, 1)])
def test_lowrank_block_tensor_cores_vs_emulation(nrem, rank, k):
    rng = np.random.default_rng(nrem + rank + k)
    W = rng.standard_normal((nrem, rank))
    H = rng.uniform(0.5, 2.0, rank)
    X = rng.standard_normal((nrem, k))
    Y = rng.standard_normal((nrem, k))
    out = P.lowrank_block_run(W, H, X, Y, tensor=True)
    Wb = bf16(W)
    T = ((Wb.T @ bf16(X)).astype(np.float32) * H.astype(np.float32)[:, None]).astype(np.float64)
    Tb = bf16(T)
    ref = Y + Wb @ Tb
    scale = np.abs(Wb) @ np.abs(Tb)
    err = np.abs(out - ref)
    # FP32 accumulation over nrem terms, plus a possible BF16 flip of one T entry per term
    bound = 1e-5 * (np.abs(Wb.T) @ np.abs(bf16(X))).max() * np.abs(Wb).max() * rank + BF16_EPS * scale
    assert (err <= bound).all(), float((err / np.maximum(bound, 1e-300)).max())
    assert np.median(err / np.maximum(scale, 1e-300)) < 1e-5  # most entries: FP32 accumulation only


@pytest.mark.parametrize("nrem,rank,k", [(1000, 20, 64), (517, 37, 13), (300, 128, 2)])
def test_lowrank_block_fp64_vs_numpy(nrem, rank, k):
    rng = np.random.default_rng(7 * nrem + rank + k)
    W = rng.standard_normal((nrem, rank))
    H = rng.uniform(0.5, 2.0, rank)
    X = rng.standard_normal((nrem, k))
    Y = rng.standard_normal((nrem, k))
    out = P.lowrank_block_run(W, H, X, Y, tensor=False)
    ref = Y + W @ (H[:, None] * (W.T @ X))
    assert np.abs(out - ref).max() <= 1e-13 * (np.abs(W) @ (H[:, None] * np.abs(W.T) @ np.abs(X))).max()


def amsed_system(precision, grid=128):
    A = P.CSRMatrix.laplacian(grid, grid, 1)
    H = P.HostAmsed(A, precision=precision, levels=3, lanczos_steps=64, low_rank=32, lowrank_type=0, reorder=0)
    S = P.DeviceSystem(A)
    S.attach(H)
    return A, H, S


def test_block_apply_fp64_equals_single_apply():
    A, H, S = amsed_system(P.PRISM_FP64)
    assert H.info()["ranks"].max() > 0, "the case must exercise the low-rank correction"
    V = np.random.default_rng(1).standard_normal((64, A.n))
    out = S.apply_batched(V)
    for c in (0, 17, 63):
        one = S.apply(V[c])
        assert np.abs(out[c] - one).max() <= 1e-12 * np.abs(one).max(), c
    # a ragged block
    out5 = S.apply_batched(V[:5])
    assert np.abs(out5 - out[:5]).max() <= 1e-12 * np.abs(out[:5]).max()


def test_block_apply_fp32_tensor_lowrank_within_bf16():
    A, H, S = amsed_system(P.PRISM_FP32)
    V = np.random.default_rng(2).standard_normal((64, A.n))
    out = S.apply_batched(V)
    for c in (0, 31, 63):
        one = S.apply(V[c])  # same FP32 factor values, FP64 low-rank products
        # the low-rank term is a part of the result; its BF16 operands perturb it by ~2^-8
        assert np.abs(out[c] - one).max() <= 8 * BF16_EPS * np.abs(one).max(), c
        assert np.isfinite(out[c]).all()


def test_block_fcg_amsed_fp64_vs_single_solves():
    A, H, S = amsed_system(P.PRISM_FP64, grid=96)
    B = np.random.default_rng(3).standard_normal((8, A.n))
    X, sts = S.solve_batched(B, tol=1e-10, max_iter=500)
    for c in range(0, 8, 3):
        x1, st1 = S.solve(B[c], tol=1e-10, max_iter=500)
        assert abs(sts[c].num_iter - st1.num_iter) <= 1 and sts[c].converged
        if sts[c].num_iter == st1.num_iter:
            assert np.abs(X[c] - x1).max() <= 1e-10 * np.abs(x1).max()


def test_block_fcg_amsed_fp32_tensor_lowrank_converges():
    A, H, S = amsed_system(P.PRISM_FP32, grid=96)
    B = np.random.default_rng(4).standard_normal((16, A.n))
    X, sts = S.solve_batched(B, tol=1e-10, max_iter=500)
    _, st1 = S.solve(B[0], tol=1e-10, max_iter=500)
    for c, st in enumerate(sts):
        assert st.converged and st.true_rel_residual < 1e-9, c
        # the BF16 low-rank term is a coarser preconditioner: measured 58 -> 63 iterations on
        # this case; the flexible outer loop keeps the tolerance
        assert st.num_iter <= int(1.15 * st1.num_iter) + 2, (c, st.num_iter, st1.num_iter)
