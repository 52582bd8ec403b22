"""Device numeric refactorisation (prism_refactor) of IC and ILDLT factors,
under every sweep layout (PRISM_SWEEP_KERNEL = global | slab | stream).

* With the values the factor was built from, the device factor equals the
  host factor (itself bit-exact with the compiled reference) to the last bit,
  and the apply is unchanged to the last bit.
* With new values on the same pattern, the device factor equals the oracle's
  fixed-pattern refactorisation (orc_refactor: the reference's setup with the
  drop test replaced by the pattern) to the last bit; the apply then matches
  the oracle's apply with that factor within 1e-12 (double arithmetic) or
  1e-5 relative 2-norm (the single-precision apply), and FCG converges.
* A matrix that is not positive definite is reported as the host reports it.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import prispack_b200 as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

CASES = [(P.PRECOND_IC, P.PRISM_FP64), (P.PRECOND_IC, P.PRISM_FP32), (P.PRECOND_IC, P.PRISM_FP32_APPLY),
         (P.PRECOND_ILDLT, P.PRISM_FP64), (P.PRECOND_ILDLT, P.PRISM_FP32)]


def _set_env(**kv):
    old = {k: os.environ.get(k) for k in kv}
    os.environ.update(kv)
    return old


def _restore_env(old):
    for k, v in old.items():
        if v is None:
            del os.environ[k]
        else:
            os.environ[k] = v


@pytest.fixture(params=["global", "slab", "stream"])
def layout(request):
    """The sweep kernel, unpaired (a paired sweep is tuned again unpaired at the first
    refactorisation: test_refactor_of_paired_sweeps)."""
    old = _set_env(PRISM_SWEEP_KERNEL=request.param, PRISM_STREAM_PAIR="0")
    yield request.param
    _restore_env(old)


def new_values(A, seed=5):
    """Same pattern, new SPD values: off-diagonal entries scaled by U[0.5, 1], diagonal raised."""
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    v = A.val.copy()
    off = rows != A.col
    # a symmetric scaling: one factor per unordered pair (i, j)
    key = np.minimum(rows, A.col).astype(np.int64) * A.n + np.maximum(rows, A.col)
    uniq, inv = np.unique(key, return_inverse=True)
    scale = rng.uniform(0.5, 1.0, len(uniq))[inv]
    v[off] *= scale[off]
    v[~off] *= 1.25
    return v


def oracle_precond(kind, n, rp, ci, lv, D):
    return orc.Precond(kind, n, (rp, ci, lv), diag=D if kind == P.PRECOND_ILDLT else None)


@pytest.mark.parametrize("kind,precision", CASES)
def test_refactor_with_the_same_values_is_bit_identical(layout, kind, precision):
    A = P.CSRMatrix.laplacian(14, 12, 10)
    S = P.DeviceSystem(A)
    S.set_precond(kind, tol=1e-3, precision=precision)
    v = np.random.default_rng(1).standard_normal(A.n)
    before = S.apply(v)
    rp, ci, val, d = S.precond_factor(0)
    S.refactor()
    rp2, ci2, val2, d2 = S.precond_factor(0)
    assert np.array_equal(rp2, rp) and np.array_equal(ci2, ci)
    assert np.array_equal(val2, val)
    if kind == P.PRECOND_ILDLT:
        assert np.array_equal(d2, d)
    assert np.array_equal(S.apply(v), before)


@pytest.mark.parametrize("kind,precision", CASES)
def test_refactor_with_new_values_matches_the_oracle(layout, kind, precision):
    A = P.CSRMatrix.laplacian(14, 12, 10)
    S = P.DeviceSystem(A)
    S.set_precond(kind, tol=1e-3, precision=precision)
    rp, ci, _, _ = S.precond_factor(0)
    val2 = new_values(A)
    S.update_values(val2)
    S.refactor()
    single = precision != P.PRISM_FP64
    rc, lv, D = orc.refactor(kind, A.rowptr, A.col, val2, rp, ci, single=single)
    assert rc == 0
    _, _, dv, dd = S.precond_factor(0)
    assert np.array_equal(dv, lv)
    if kind == P.PRECOND_ILDLT:
        assert np.array_equal(dd, D)
    v = np.random.default_rng(2).standard_normal(A.n)
    got = S.apply(v)
    ref = v.copy()
    orc_pre = oracle_precond(kind, A.n, rp, ci, lv, D)
    ref = orc_pre.apply(ref)
    if precision == P.PRISM_FP32_APPLY:
        assert np.linalg.norm(got - ref) <= 1e-5 * np.linalg.norm(ref)
    else:
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    b = np.random.default_rng(3).standard_normal(A.n)
    x, st = S.solve(b, tol=1e-10, max_iter=500)
    assert st.converged and st.true_rel_residual < 1e-9


def test_refactor_reaches_the_block_sweeps():
    A = P.CSRMatrix.laplacian(24, 20, 1)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3, precision=P.PRISM_FP32)
    V = np.random.default_rng(4).standard_normal((5, A.n))
    S.apply_batched(V)  # level-order copies built from the host factor
    S.update_values(new_values(A, seed=9))
    S.refactor()
    out = S.apply_batched(V)
    for c in range(5):
        one = S.apply(V[c])
        assert np.abs(out[c] - one).max() <= 1e-12 * np.abs(one).max(), c


def test_refactor_reports_what_the_host_reports():
    A = P.CSRMatrix.laplacian(10, 10, 1)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3)
    S.update_values(-A.val)
    with pytest.raises(P.PrismError) as e:
        S.refactor()
    assert e.value.status == 4  # PRISM_ERR_NOT_SPD
    # the handle stays usable: the right values and a refactorisation bring it back
    S.update_values(A.val)
    S.refactor()
    x, st = S.solve(np.ones(A.n), tol=1e-10)
    assert st.converged


def test_refactor_is_refused_where_it_does_not_exist():
    A = P.CSRMatrix.laplacian(10, 10, 1, 0.3, 0.0, 0.0)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_ILUT, tol=1e-3, lfill=10)
    with pytest.raises(P.PrismError) as e:
        S.refactor()
    assert e.value.status == 9  # PRISM_ERR_UNSUPPORTED


@pytest.mark.parametrize("kind,precision", [(P.PRECOND_IC, P.PRISM_FP64), (P.PRECOND_ILDLT, P.PRISM_FP32_APPLY)])
def test_refactor_of_paired_sweeps(kind, precision):
    """Streamed sweeps running paired (wavefront pairing): the first refactorisation tunes
    them again unpaired, whose value maps it fills; the factor is the oracle's bit for bit
    and the apply matches the oracle's as for unpaired sweeps."""
    old = _set_env(PRISM_SWEEP_KERNEL="stream", PRISM_STREAM_PAIR="2")
    try:
        A = P.CSRMatrix.laplacian(14, 12, 10)
        S = P.DeviceSystem(A)
        S.set_precond(kind, tol=1e-3, precision=precision)
        assert S.sweep_order(0).paired and S.sweep_order(1).paired
        rp, ci, _, _ = S.precond_factor(0)
        val2 = new_values(A, seed=12)
        S.update_values(val2)
        S.refactor()
        assert not S.sweep_order(0).paired and not S.sweep_order(1).paired
        rc, lv, D = orc.refactor(kind, A.rowptr, A.col, val2, rp, ci, single=precision != P.PRISM_FP64)
        assert rc == 0
        _, _, dv, dd = S.precond_factor(0)
        assert np.array_equal(dv, lv)
        v = np.random.default_rng(2).standard_normal(A.n)
        got = S.apply(v)
        ref = oracle_precond(kind, A.n, rp, ci, lv, D).apply(v.copy())
        if precision == P.PRISM_FP32_APPLY:
            assert np.linalg.norm(got - ref) <= 1e-5 * np.linalg.norm(ref)
        else:
            assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
        x, st = S.solve(np.random.default_rng(3).standard_normal(A.n), tol=1e-10, max_iter=500)
        assert st.converged and st.true_rel_residual < 1e-9
    finally:
        _restore_env(old)
