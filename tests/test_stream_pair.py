"""Wavefront pairing of a triangular sweep (pair_sweep, prism_stream_sweep_pair),
checked on the host: a row on an odd wavefront 2R+1 has its dependencies on
wavefront 2R substituted by their own rows, so that

    T^{-1} b = T'^{-1} (b - M b)

for the paired sweep T' and the right-hand side map M, and every row's
wavefront in T' is half (rounded down) its wavefront in T.  Plain forward /
backward substitution (the sequential loops of IncompleteLDLT.cpp:188-233 /
IncompleteCholesky.cpp:249-295) solves both sides in double."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P
from test_stream_layout import random_triangular, substitute


def levels(rowptr, col, lower):
    n = len(rowptr) - 1
    lev = np.zeros(n, np.int64)
    rows = range(n) if lower else range(n - 1, -1, -1)
    for r in rows:
        deps = col[rowptr[r]:rowptr[r + 1]]
        lev[r] = 1 + lev[deps].max() if len(deps) else 0
    return lev


def apply_map(mptr, mdep, mcoef, b):
    out = b.copy()
    for r in range(len(mptr) - 1):
        for q in range(mptr[r], mptr[r + 1]):
            out[r] -= mcoef[q] * b[mdep[q]]
    return out


@pytest.mark.parametrize("op", [0, 1, 2, 3])
@pytest.mark.parametrize("lower", [True, False])
def test_paired_sweep_solves_the_same_system(op, lower):
    rng = np.random.default_rng(11 + op + 4 * lower)
    n = 400
    rp, ci, v = random_triangular(n, lower, rng)
    d = rng.uniform(1.5, 3.0, n)
    prow, pcol, pval, mptr, mdep, mcoef = P.stream_sweep_pair(rp, ci, v, diag=d, op=op, lower=lower,
                                                              precision=P.PRISM_FP64)
    # gather form, dependencies in increasing order on the sweep's side of the diagonal
    for r in range(n):
        deps = pcol[prow[r]:prow[r + 1]]
        assert np.all(np.diff(deps.astype(np.int64)) > 0)
        assert np.all(deps < r) if lower else np.all(deps > r)
    lev, plev = levels(rp, ci, lower), levels(prow, pcol, lower)
    assert np.array_equal(plev, lev // 2)
    # only rows on odd wavefronts carry a map, one entry per dependency on the wavefront before
    for r in range(n):
        deps = ci[rp[r]:rp[r + 1]]
        want = sorted(int(j) for j in deps if lev[r] % 2 == 1 and lev[j] == lev[r] - 1)
        assert sorted(mdep[mptr[r]:mptr[r + 1]].tolist()) == want
    b = rng.standard_normal(n)
    x = substitute(rp, ci, v, d, op, lower, b)
    xp = substitute(prow, pcol, pval, d, op, lower, apply_map(mptr, mdep, mcoef, b))
    assert np.abs(xp - x).max() <= 1e-12 * np.abs(x).max()


def test_paired_ic_factor_of_poisson():
    """IC(1e-3) of 3D Poisson 10^3: both sweeps paired, the wavefronts halved, the solve kept."""
    A = P.CSRMatrix.laplacian(10, 10, 10)
    F = P.HostFactor(A, P.PRECOND_IC, tol=1e-3)
    rp, ci, val = F.arrays()[:3]  # L^T by rows, diagonal first
    n = A.n
    Lt = np.zeros((n, n))
    rows = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
    Lt[rows, ci] = val
    L = Lt.T
    # lower sweep in gather form: row r depends on L[r, j], j < r; op 0 divides by L[r, r]
    lrp, lci, lv = [0], [], []
    for r in range(n):
        js = np.nonzero(L[r, :r])[0]
        lci += js.tolist()
        lv += L[r, js].tolist()
        lrp.append(len(lci))
    lrp, lci, lv, d = np.array(lrp, np.uint32), np.array(lci, np.uint32), np.array(lv), np.diag(L).copy()
    prow, pcol, pval, mptr, mdep, mcoef = P.stream_sweep_pair(lrp, lci, lv, diag=d, op=0, lower=True,
                                                              precision=P.PRISM_FP64)
    lev, plev = levels(lrp, lci, True), levels(prow, pcol, True)
    assert plev.max() == lev.max() // 2
    b = np.random.default_rng(3).standard_normal(n)
    x = np.linalg.solve(L, b)
    xp = substitute(prow, pcol, pval, d, 0, True, apply_map(mptr, mdep, mcoef, b))
    assert np.abs(xp - x).max() <= 1e-11 * np.abs(x).max()


def test_paired_sweep_with_single_precision_values():
    """Values rounded to float (the single-precision sweeps): the paired solve stays within
    float rounding of the unpaired one."""
    rng = np.random.default_rng(5)
    rp, ci, v = random_triangular(300, True, rng)
    d = rng.uniform(1.5, 3.0, 300)
    prow, pcol, pval, mptr, mdep, mcoef = P.stream_sweep_pair(rp, ci, v, diag=d, op=0, lower=True,
                                                              precision=P.PRISM_FP32)
    assert np.array_equal(pval.astype(np.float32).astype(np.float64), pval)
    b = rng.standard_normal(300)
    x = substitute(rp, ci, v.astype(np.float32).astype(np.float64), d, 0, True, b)
    xp = substitute(prow, pcol, pval, d, 0, True, apply_map(mptr, mdep, mcoef, b))
    assert np.abs(xp - x).max() <= 1e-5 * np.abs(x).max()


def test_pairing_does_not_depend_on_host_threads(monkeypatch):
    """Large sweeps are paired on several host threads, rows in contiguous chunks, and
    assembled in row order: one thread and several give the same arrays to the bit."""
    n = 90000
    offs = np.array([1, 7, 50, 2500])
    rows = np.repeat(np.arange(n), len(offs))
    cols = rows - np.tile(offs, n)
    keep = cols >= 0
    rows, cols = rows[keep], cols[keep]
    rp = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.uint32)
    ci = cols.astype(np.uint32)
    v = np.random.default_rng(8).uniform(-0.2, 0.2, len(ci))
    d = np.random.default_rng(9).uniform(1.5, 3.0, n)
    got = []
    for threads in ("1", "6"):
        monkeypatch.setenv("PRISM_LAYOUT_THREADS", threads)
        got.append(P.stream_sweep_pair(rp, ci, v, diag=d, op=0, lower=True, precision=P.PRISM_FP64))
    for a, b in zip(*got):
        assert np.array_equal(a, b)
