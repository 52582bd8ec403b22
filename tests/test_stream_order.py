"""The streamed sweep kernel's summation order, checked on the host.

prism_stream_sweep_order exports, per row, the order in which the kernel
sums its entries; oracle.sweep_ordered restates that arithmetic in plain C.
The library's own host replay of the kernel (prism_selftest_stream_layout,
which decodes the round records exactly as the kernel does) must equal the
oracle bit for bit, and both must agree with plain substitution in stored
order (the reference's sweeps, IncompleteLDLT.cpp:188-233) within rounding.
The exported order must also be a permutation of each row's entries plus
zero-coefficient padding, so that the kernel computes the same sweep."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P
from oracle import oracle as orc
from test_stream_layout import random_triangular, substitute

SINGLE = {P.PRISM_FP32_APPLY: True, P.PRISM_FP32: False, P.PRISM_FP64: False}


def bitwise_equal(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint64), np.ascontiguousarray(b).view(np.uint64))


@pytest.mark.parametrize("precision", [P.PRISM_FP32_APPLY, P.PRISM_FP32, P.PRISM_FP64])
@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_replay_equals_ordered_oracle(precision, lower, op):
    rng = np.random.default_rng(300 + 10 * op + lower)
    n = 900
    rp, ci, v = random_triangular(n, lower, rng, near=10, far=3, long_rows=(37, 400, 650))
    if precision != P.PRISM_FP64:
        v = v.astype(np.float32).astype(np.float64)
    d = rng.uniform(1.0, 2.0, n)
    b = rng.standard_normal(n)
    want = substitute(rp, ci, v, d, op, lower, b)
    for ctas in (1, 5, 28):
        o = P.stream_sweep_order(rp, ci, v, diag=d, op=op, lower=lower, precision=precision, num_ctas=ctas)
        ref = orc.sweep_ordered(o, b, diag=d, op=op, lower=lower, single=SINGLE[precision])
        rep = P.selftest_stream_layout(rp, ci, v, b, diag=d, op=op, lower=lower, precision=precision,
                                       num_ctas=ctas, rows_per_cta=0)
        assert bitwise_equal(rep, ref)
        tol = 1e-4 if SINGLE[precision] else 1e-12
        assert np.abs(ref - want).max() <= tol * np.abs(want).max()


def test_order_is_a_permutation_of_each_row():
    rng = np.random.default_rng(8)
    n = 2000
    rp, ci, v = random_triangular(n, True, rng, near=12, far=4, long_rows=(100, 1500))
    for precision in (P.PRISM_FP32_APPLY, P.PRISM_FP64):
        o = P.stream_sweep_order(rp, ci, v, op=2, lower=True, precision=precision, num_ctas=16)
        vv = v.astype(np.float32).astype(np.float64) if precision != P.PRISM_FP64 else v
        for r in range(n):
            deps = list(o.edep[o.eptr[r]:o.eptr[r + 1]]) + list(o.kdep[o.kptr[r]:o.kptr[r + 1]])
            coef = list(o.ecoef[o.eptr[r]:o.eptr[r + 1]]) + list(o.kcoef[o.kptr[r]:o.kptr[r + 1]])
            got = sorted((d, c) for d, c in zip(deps, coef) if d != P.SweepOrder.PAD)
            want = sorted(zip(ci[rp[r]:rp[r + 1]].tolist(), vv[rp[r]:rp[r + 1]].tolist()))
            assert got == want
            assert all(c == 0.0 for d, c in zip(deps, coef) if d == P.SweepOrder.PAD)
            # whole groups of four positions
            assert (o.eptr[r + 1] - o.eptr[r]) % 4 == 0 and (o.kptr[r + 1] - o.kptr[r]) % 4 == 0


def test_late_entries_are_few_on_a_3d_factor():
    """On an IC factor of 3D Poisson most of a row's entries are summed ahead of
    their round: the late ones (slab rows of the kStreamLate = 3 rounds just
    before) are under a third of them."""
    A = P.CSRMatrix.laplacian(16, 16, 16)
    F = P.HostFactor(A, P.PRECOND_IC, tol=1e-3)
    rp, ci, v, _ = F.arrays(0)
    n = A.n
    rows = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
    off = ci.astype(np.int64) != rows
    urp = np.concatenate([[0], np.cumsum(np.bincount(rows[off], minlength=n))]).astype(np.uint32)
    o = P.stream_sweep_order(urp, ci[off], v[off], diag=v[rp[:-1]], op=0, lower=False,
                             precision=P.PRISM_FP32_APPLY, num_ctas=8)
    late = int((o.kdep != P.SweepOrder.PAD).sum())
    early = int((o.edep != P.SweepOrder.PAD).sum())
    assert late + early == int(off.sum())
    assert late < 0.3 * (late + early)
