"""The streamed sweep kernel against the oracle, bit for bit.

The kernel sums each row in its own order: the "early" entries in four
interleaved fused multiply-add chains, then the "late" ones (the slab's rows of
the three rounds just before) one by one (prism_stream_sweep_order states the
order).
oracle.sweep_ordered restates that arithmetic in plain C from the exported
order alone, so the GPU results must equal it to the last bit, in float for
the single-precision apply (PRISM_FP32_APPLY) and in double otherwise; the
reference-order sweeps (substitution in stored order, IncompleteLDLT.cpp:
188-233) agree within rounding.  The whole AMSED apply adds double-precision
coupling and low-rank products whose summation order differs from the
oracle's, so it is compared within a stated tolerance."""
from __future__ import annotations

import os

import numpy as np
import pytest

import prispack_b200 as P
from oracle import oracle as orc
from test_stream_layout import random_triangular, substitute

pytestmark = pytest.mark.gpu

SINGLE = {P.PRISM_FP32_APPLY: True, P.PRISM_FP32: False, P.PRISM_FP64: False}


def bitwise_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


@pytest.mark.parametrize("precision", [P.PRISM_FP32_APPLY, P.PRISM_FP32, P.PRISM_FP64])
@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_random_sweeps_match_ordered_oracle_bitwise(precision, lower, op):
    rng = np.random.default_rng(1000 + 10 * op + lower)
    n = 3000
    rp, ci, v = random_triangular(n, lower, rng, near=10, far=3, long_rows=(37, 1400, 2650))
    if precision != P.PRISM_FP64:
        v = v.astype(np.float32).astype(np.float64)
    d = rng.uniform(1.0, 2.0, n)
    b = rng.standard_normal(n)
    want = substitute(rp, ci, v, d, op, lower, b)
    for ctas in (1, 7, 64, 148):
        order = P.stream_sweep_order(rp, ci, v, diag=d, op=op, lower=lower, precision=precision, num_ctas=ctas)
        ref = orc.sweep_ordered(order, b, diag=d, op=op, lower=lower, single=SINGLE[precision])
        got = P.stream_sweep_run(rp, ci, v, b, diag=d, op=op, lower=lower, precision=precision, num_ctas=ctas)
        assert bitwise_equal(got, ref), (ctas, float(np.abs(got - ref).max()))
        tol = 1e-4 if SINGLE[precision] else 1e-12
        assert np.abs(got - want).max() <= tol * np.abs(want).max()


@pytest.mark.parametrize("precision", [P.PRISM_FP32_APPLY, P.PRISM_FP64])
@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_paired_random_sweeps_match_ordered_oracle_bitwise(precision, lower, op):
    """Wavefront pairing (prism_stream_sweep_pair): the paired sweep through the kernel
    equals the ordered oracle bit for bit on the mapped right-hand side, and the paired
    solve equals the unpaired substitution within rounding."""
    rng = np.random.default_rng(2000 + 10 * op + lower)
    n = 3000
    rp, ci, v = random_triangular(n, lower, rng, near=10, far=3, long_rows=(37, 1400, 2650))
    if precision != P.PRISM_FP64:
        v = v.astype(np.float32).astype(np.float64)
    d = rng.uniform(1.0, 2.0, n)
    b = rng.standard_normal(n)
    want = substitute(rp, ci, v, d, op, lower, b)
    prow, pcol, pval, mptr, mdep, mcoef = P.stream_sweep_pair(rp, ci, v, diag=d, op=op, lower=lower,
                                                              precision=precision)
    bp = orc.pair_rhs(mptr, mdep, mcoef, b)
    for ctas in (1, 7, 148):
        order = P.stream_sweep_order(prow, pcol, pval, diag=d, op=op, lower=lower, precision=precision,
                                     num_ctas=ctas)
        ref = orc.sweep_ordered(order, bp, diag=d, op=op, lower=lower, single=SINGLE[precision])
        got = P.stream_sweep_run(prow, pcol, pval, bp, diag=d, op=op, lower=lower, precision=precision,
                                 num_ctas=ctas)
        assert bitwise_equal(got, ref), (ctas, float(np.abs(got - ref).max()))
        tol = 1e-4 if SINGLE[precision] else 1e-11
        assert np.abs(got - want).max() <= tol * np.abs(want).max()


@pytest.fixture(params=["0", "2"], ids=["unpaired", "paired"])
def pairing(request):
    """PRISM_STREAM_PAIR for the handles a test builds: 0 never paired, 2 paired where it fits."""
    old = os.environ.get("PRISM_STREAM_PAIR")
    os.environ["PRISM_STREAM_PAIR"] = request.param
    yield request.param == "2"
    if old is None:
        del os.environ["PRISM_STREAM_PAIR"]
    else:
        os.environ["PRISM_STREAM_PAIR"] = old


def _handle_sweep_check(S, sweep, single, rng):
    import torch
    S.set_stream(torch.cuda.current_stream().cuda_stream)  # the tensors' stream
    info = S.sweep_info(sweep)
    assert info["kernel"] == "stream"
    order = S.sweep_order(sweep)
    vin = rng.standard_normal(info["n"])
    tin = torch.tensor(vin, device="cuda")
    tout = torch.empty_like(tin)
    S.sweep_device(sweep, tin, tout, 1)
    torch.cuda.synchronize()
    got = tout.cpu().numpy()
    ref = orc.sweep_ordered(order, vin, diag=order.diag, op=order.op, lower=order.lower, single=single)
    assert bitwise_equal(got, ref), (sweep, float(np.abs(got - ref).max()))
    return order


@pytest.mark.parametrize("kind", [P.PRECOND_IC, P.PRECOND_ILDLT, P.PRECOND_ILUT])
def test_triangular_sweeps_and_apply_bitwise(kind):
    """Single-precision apply of IC / ILDLT (3D Poisson 24^3) and ILUT (3D
    convection-diffusion 20^3): each sweep, and the apply (lower then upper
    sweep), equal the kernel-order oracle bit for bit."""
    rng = np.random.default_rng(40 + kind)
    if kind == P.PRECOND_ILUT:
        A = P.CSRMatrix.convection_diffusion(20, 20, 20, 10.0, 5.0, 2.5)
        kw = dict(tol=1e-3, lfill=20)
    else:
        A = P.CSRMatrix.laplacian(24, 24, 24)
        kw = dict(tol=1e-3)
    S = P.DeviceSystem(A)
    S.set_precond(kind, precision=P.PRISM_FP32_APPLY, **kw)
    lo = _handle_sweep_check(S, 0, True, rng)
    up = _handle_sweep_check(S, 1, True, rng)
    v = rng.standard_normal(A.n)
    t = orc.sweep_ordered(lo, v, diag=lo.diag, op=lo.op, lower=lo.lower, single=True)
    ref = orc.sweep_ordered(up, t, diag=up.diag, op=up.op, lower=up.lower, single=True)
    assert bitwise_equal(S.apply(v), ref)


@pytest.mark.parametrize("precision", [P.PRISM_FP32, P.PRISM_FP64])
def test_double_arithmetic_streamed_sweeps_bitwise(precision):
    """The double-arithmetic precisions, streamed layout forced on an IC factor."""
    import os
    rng = np.random.default_rng(77)
    A = P.CSRMatrix.laplacian(20, 20, 20)
    os.environ["PRISM_SWEEP_KERNEL"] = "stream"
    try:
        S = P.DeviceSystem(A)
        S.set_precond(P.PRECOND_IC, tol=1e-3, precision=precision)
    finally:
        del os.environ["PRISM_SWEEP_KERNEL"]
    for sw in (0, 1):
        _handle_sweep_check(S, sw, False, rng)


AMSED_OPTS = dict(levels=3, lanczos_steps=32, low_rank=16, lowrank_type=0, reorder=0)


def test_amsed_level_sweeps_bitwise_and_apply_against_oracle(pairing):
    """AMSED/MSLR on 3D Poisson 32^3 with the single-precision apply, the level
    sweeps paired or not: every level's block sweeps (a paired one with its
    right-hand side map) equal the kernel-order oracle bit for bit; the whole
    apply equals the oracle's AMSED apply (orc_amsed_apply with kernel-order
    float sweeps, double elsewhere) to within 1e-6 relative in the max norm,
    the room left for the coupling and low-rank products, which sum in
    another order on the device (a last-bit difference there can move a float
    rounding in a later sweep)."""
    rng = np.random.default_rng(55)
    A = P.CSRMatrix.laplacian(32, 32, 32)
    F = P.HostAmsed(A, precision=P.PRISM_FP32_APPLY, **AMSED_OPTS)
    S = P.DeviceSystem(A)
    S.attach(F)
    nlev = int(F.info()["nlev"])
    orders = [_handle_sweep_check(S, sw, True, rng) for sw in range(2 * nlev)]
    assert all(o.paired == pairing for o in orders)
    O = orc.Amsed(F)
    O.use_sweep_orders(orders, single=True)
    for seed in (1, 2, 3):
        v = np.random.default_rng(seed).standard_normal(A.n)
        got, ref = S.apply(v), O.apply(v)
        assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()


def test_amsed_fp32_apply_solve_matches_oracle_fcg(pairing):
    """FCG + AMSED with the single-precision apply on the device against the
    oracle's FCG with the same (kernel-order, float-sweep) AMSED apply: the
    same iteration count within 1 and solutions within 1e-9 relative."""
    A = P.CSRMatrix.laplacian(32, 32, 32)
    F = P.HostAmsed(A, precision=P.PRISM_FP32_APPLY, **AMSED_OPTS)
    S = P.DeviceSystem(A)
    S.attach(F)
    nlev = int(F.info()["nlev"])
    O = orc.Amsed(F)
    O.use_sweep_orders([S.sweep_order(sw) for sw in range(2 * nlev)], single=True)
    b = np.random.default_rng(9).standard_normal(A.n)
    x, st = S.solve(b, tol=1e-10, max_iter=500)
    xo, ito, _, _ = orc.cg(A.rowptr, A.col, A.val, b, O.precond(), tol=1e-10, maxit=500)
    assert st.converged and abs(st.num_iter - ito) <= 1
    assert np.linalg.norm(x - xo) <= 1e-9 * np.linalg.norm(xo)
