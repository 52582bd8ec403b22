"""Streamed round layout of the triangular sweep kernel (k_sweep_stream),
checked on the host: prism_selftest_stream_layout builds the slabs, rounds,
value slots and round records, replays the kernel's decoding of every record
(bounds, which value each slot holds when it is read, no wait on a later
round), and solves the sweep; the result must equal a plain forward /
backward substitution (the sequential loops of IncompleteLDLT.cpp:188-233 /
IncompleteCholesky.cpp:249-295)."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P


def random_triangular(n, lower, rng, near=6, far=3, long_rows=()):
    """Gather-form triangular pattern: row r lists dependencies on one side of
    the diagonal, mostly close to r (stencil-like), a few far away."""
    rowptr, col = [0], []
    for r in range(n):
        cand = set()
        pool = np.arange(0, r) if lower else np.arange(r + 1, n)
        if len(pool):
            k = min(len(pool), near)
            close = pool[-k:] if lower else pool[:k]
            cand.update(rng.choice(close, size=rng.integers(0, k + 1), replace=False).tolist())
            cand.update(rng.choice(pool, size=min(len(pool), rng.integers(0, far + 1)), replace=False).tolist())
            if r in long_rows:
                cand.update(rng.choice(pool, size=min(len(pool), 70), replace=False).tolist())
        c = sorted(cand)
        col += c
        rowptr.append(len(col))
    col = np.array(col, np.uint32)
    val = rng.uniform(-0.3, 0.3, len(col))
    return np.array(rowptr, np.uint32), col, val


def substitute(rowptr, col, val, diag, op, lower, b):
    n = len(rowptr) - 1
    x = np.zeros(n)
    rows = range(n) if lower else range(n - 1, -1, -1)
    for r in rows:
        s = float(np.dot(val[rowptr[r]:rowptr[r + 1]], x[col[rowptr[r]:rowptr[r + 1]]]))
        if op == 0:
            x[r] = (b[r] - s) / diag[r]
        elif op == 1:
            x[r] = (b[r] - s) * diag[r]
        elif op == 2:
            x[r] = b[r] - s
        else:
            x[r] = b[r] / diag[r] - s
    return x


@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_replay_matches_substitution(lower, op):
    rng = np.random.default_rng(100 + op + 10 * lower)
    n = 701
    rp, ci, v = random_triangular(n, lower, rng, long_rows=(37, 400, 650))
    diag = rng.uniform(1.0, 2.0, n)
    b = rng.standard_normal(n)
    want = substitute(rp, ci, v, diag, op, lower, b)
    for ctas in (1, 3, 7, 32):
        got = P.selftest_stream_layout(rp, ci, v, b, diag=diag, op=op, lower=lower, num_ctas=ctas)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)


def test_replay_fp32_values():
    rng = np.random.default_rng(7)
    n = 333
    rp, ci, v = random_triangular(n, True, rng)
    b = rng.standard_normal(n)
    want = substitute(rp, ci, v.astype(np.float32).astype(np.float64), None, 2, True, b)
    got = P.selftest_stream_layout(rp, ci, v, b, op=2, lower=True, precision=P.PRISM_FP32, num_ctas=5)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)


def test_replay_ic_factor_of_poisson():
    """The IC factor of a 3D Poisson problem, both sweeps, slabs of uneven size."""
    A = P.CSRMatrix.laplacian(12, 11, 10)
    F = P.HostFactor(A, P.PRECOND_IC, tol=1e-3)
    rp, ci, v, d = F.arrays(0)  # rows of L^T, diagonal first
    n = A.n
    rp = rp.astype(np.int64)
    # lower sweep (gather form): row j depends on i < j through L^T(i, j)
    rows = np.repeat(np.arange(n), np.diff(rp))
    off = ci.astype(np.int64) != rows
    src, dst, w = rows[off], ci.astype(np.int64)[off], v[off]
    o = np.lexsort((src, dst))
    src, dst, w = src[o], dst[o], w[o]
    lrp = np.zeros(n + 1, np.int64)
    np.add.at(lrp, dst + 1, 1)
    lrp = np.cumsum(lrp)
    diag = v[rp[:-1]]
    b = np.random.default_rng(3).standard_normal(n)
    want = substitute(lrp, src, w, diag, 0, True, b)
    got = P.selftest_stream_layout(lrp, src, w, b, diag=diag, op=0, lower=True, num_ctas=9, rows_per_cta=150)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-13)
    # upper sweep (gather form): row i depends on j > i through L^T(i, j)
    ucol, uval = ci[off], v[off]
    urp = np.concatenate([[0], np.cumsum(np.bincount(rows[off], minlength=n))]).astype(np.uint32)
    want = substitute(urp, ucol, uval, diag, 0, False, b)
    got = P.selftest_stream_layout(urp, ucol, uval, b, diag=diag, op=0, lower=False, num_ctas=9, rows_per_cta=150)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-13)


def test_layout_rejects_what_it_cannot_encode():
    rng = np.random.default_rng(5)
    rp, ci, v = random_triangular(100, True, rng)
    with pytest.raises(P.PrismError):  # slabs that do not cover the rows
        P.selftest_stream_layout(rp, ci, v, np.ones(100), op=2, num_ctas=2, rows_per_cta=10)
    with pytest.raises(P.PrismError):  # a dependency on the wrong side of the diagonal
        P.selftest_stream_layout(rp, ci, v, np.ones(100), op=2, lower=False, num_ctas=2)


@pytest.mark.parametrize("ctas,rows", [(40, None), (63, 80), (3, None)])
def test_replay_many_slabs_and_slot_reuse(ctas, rows):
    """Many small slabs: most dependencies are halo rows, slots are reused often."""
    rng = np.random.default_rng(ctas)
    n = 5000
    rp, ci, v = random_triangular(n, True, rng, near=12, far=2)
    d = rng.uniform(1.0, 2.0, n)
    b = rng.standard_normal(n)
    want = substitute(rp, ci, v, d, 3, True, b)
    got = P.selftest_stream_layout(rp, ci, v, b, diag=d, op=3, lower=True, num_ctas=ctas, rows_per_cta=rows)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)
    rp, ci, v = random_triangular(n, False, np.random.default_rng(ctas + 1), near=12, far=2)
    want = substitute(rp, ci, v, d, 3, False, b)
    got = P.selftest_stream_layout(rp, ci, v, b, diag=d, op=3, lower=False, num_ctas=ctas, rows_per_cta=rows)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)


def test_replay_block_diagonal_slabs_follow_the_blocks():
    """Slab boundaries chosen by the layout (rows_per_cta = 0) on a block-diagonal
    factor: blocks of uneven size, solved exactly as one sweep."""
    rng = np.random.default_rng(21)
    sizes = [700, 1300, 400, 900]
    rps, cis, vs, off = [np.zeros(1, np.uint32)], [], [], 0
    for m in sizes:
        rp, ci, v = random_triangular(m, True, rng, near=10, far=2)
        rps.append(rp[1:] + rps[-1][-1])
        cis.append(ci + off)
        vs.append(v)
        off += m
    rp, ci, v = np.concatenate(rps), np.concatenate(cis), np.concatenate(vs)
    n = off
    d = rng.uniform(1.0, 2.0, n)
    b = rng.standard_normal(n)
    want = substitute(rp, ci, v, d, 0, True, b)
    for ctas in (4, 7, 19):
        got = P.selftest_stream_layout(rp, ci, v, b, diag=d, op=0, lower=True, num_ctas=ctas, rows_per_cta=0)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)


def test_layout_does_not_depend_on_host_threads(monkeypatch):
    """The streamed layout is built slab by slab on several host threads and assembled in
    slab order: one thread and several give the same summation order and the same replay."""
    rng = np.random.default_rng(77)
    n = 6000
    rp, ci, v = random_triangular(n, True, rng, near=12, far=4, long_rows=(100, 3000))
    d = rng.uniform(1.0, 2.0, n)
    b = rng.standard_normal(n)
    got = []
    for threads in ("1", "5"):
        monkeypatch.setenv("PRISM_LAYOUT_THREADS", threads)
        o = P.stream_sweep_order(rp, ci, v, diag=d, op=0, lower=True, precision=P.PRISM_FP32_APPLY, num_ctas=40)
        x = P.selftest_stream_layout(rp, ci, v, b, diag=d, op=0, lower=True, precision=P.PRISM_FP32_APPLY,
                                     num_ctas=40)
        got.append((o, x))
    (o1, x1), (o2, x2) = got
    for f in ("eptr", "edep", "ecoef", "kptr", "kdep", "kcoef"):
        assert np.array_equal(getattr(o1, f), getattr(o2, f)), f
    assert np.array_equal(x1, x2)


@pytest.mark.parametrize("precision", [P.PRISM_FP32_APPLY, P.PRISM_FP64])
def test_capped_rounds_replay_and_respect_the_cap(precision):
    """Rounds cut short where their record would pass a byte cap (what the device layout
    does when four of its largest records would not fit the ring): the records stay within
    half of the uncapped layout's largest, and the replay still solves the sweep.  (A round
    keeps at least one row, so a cap below one row's record cannot hold.)"""
    rng = np.random.default_rng(33)
    n = 4000
    rp, ci, v = random_triangular(n, True, rng, near=24, far=6)
    d = rng.uniform(1.0, 2.0, n)
    b = rng.standard_normal(n)
    want = substitute(rp, ci, v, d, 0, True, b)
    free, rec_free = P.selftest_stream_layout_capped(rp, ci, v, b, max_round_bytes=0, diag=d, op=0,
                                                     precision=precision, num_ctas=6)
    cap = rec_free // 2 // 16 * 16
    got, rec = P.selftest_stream_layout_capped(rp, ci, v, b, max_round_bytes=cap, diag=d, op=0,
                                               precision=precision, num_ctas=6)
    assert rec <= cap
    tol = 1e-4 if precision == P.PRISM_FP32_APPLY else 1e-12
    for x in (free, got):
        assert np.abs(x - want).max() <= tol * np.abs(want).max()
