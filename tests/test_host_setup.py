"""Product host setup (model problems, incomplete factorisations, level
schedules, input validation) against the reference's golden outputs.  CPU only:
these entry points run on the host and never touch a device."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

import prispack_b200 as P

CASES = ["lap2d_8", "lap3d_6", "conv2d_16", "lap2d_64"]
KIND = {1: P.PRECOND_IC, 2: P.PRECOND_ILUT, 3: P.PRECOND_ILDLT}


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", CASES)
def test_laplacian_matches_reference(name, manifest, load_golden):
    g = load_golden(name)
    A = P.CSRMatrix.laplacian(*manifest[name]["grid"])
    assert np.array_equal(A.rowptr, g["rowptr"]) and np.array_equal(A.col, g["col"])
    assert np.array_equal(A.val, g["val"])


@pytest.mark.parametrize("name", CASES)
def test_factors_bit_exact(name, manifest, load_golden):
    """Every stored factor array equals the reference's setup() output bit for bit."""
    g = load_golden(name)
    A = P.CSRMatrix(g["rowptr"], g["col"], g["val"])
    for key, e in manifest[name]["precond"].items():
        if e.get("setup_rc") != 0:
            continue
        prec = P.PRISM_FP32 if key.endswith("fp32") else P.PRISM_FP64
        F = P.HostFactor(A, KIND[e["kind"]], tol=e["tol"], lfill=e["lfill"], precision=prec)
        rp, ci, v, d = F.arrays(0)
        assert sha(rp, ci, v) == e["f0_sha"], key
        if e["kind"] == 3:
            assert sha(d) == e["diag_sha"], key
        if e["kind"] == 2:
            rp1, ci1, v1, d1 = F.arrays(1)
            assert sha(rp1, ci1, v1) == e["f1_sha"], key
            assert sha(d1) == e["diag_sha"], key
        assert F.info()["mnnz"] == e["mnnz"], key


def _levels(rp, ci, lower):
    n = len(rp) - 1
    lev = np.zeros(n, np.int64)
    rng = range(n) if lower else range(n - 1, -1, -1)
    for i in rng:
        deps = ci[rp[i]:rp[i + 1]]
        lev[i] = lev[deps].max() + 1 if len(deps) else 0
    return int(lev.max()) + 1


@pytest.mark.parametrize("name", ["lap2d_8", "lap3d_6", "lap2d_64"])
def test_level_schedule_counts(name, load_golden):
    """The exact integer level schedule: wavefront count of the IC sweeps from the factor pattern."""
    g = load_golden(name)
    A = P.CSRMatrix(g["rowptr"], g["col"], g["val"])
    F = P.HostFactor(A, P.PRECOND_IC, tol=1e-3)
    rp, ci, v, _ = F.arrays(0)
    n = A.n
    # strictly-upper part of L^T: upper sweep deps; its transpose: lower sweep deps
    urp = np.zeros(n + 1, np.int64)
    rows, cols = [], []
    for i in range(n):
        c = ci[rp[i] + 1:rp[i + 1]]
        rows += [i] * len(c)
        cols += list(c)
        urp[i + 1] = urp[i] + len(c)
    up = _levels(urp, np.array(cols, np.int64), lower=False)
    import scipy.sparse as sp
    U = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, n))
    L = U.T.tocsr()
    lo = _levels(L.indptr, L.indices, lower=True)
    info = F.info()
    assert info["upper_levels"] == up and info["lower_levels"] == lo


def test_not_spd_reports_status():
    # shifted Laplacian: IC meets a non-positive pivot, the reference prints and stops
    A = P.CSRMatrix.laplacian(6, 6, 1, shift=5.0)
    with pytest.raises(P.PrismError) as e:
        P.HostFactor(A, P.PRECOND_IC, tol=0.0)
    assert e.value.status == 4


def test_zero_pivot_reports_status():
    rp = np.array([0, 2, 4], np.uint32)
    ci = np.array([0, 1, 0, 1], np.uint32)
    v = np.array([1.0, 1.0, 1.0, 1.0])  # singular: second pivot is 0
    A = P.CSRMatrix(rp, ci, v)
    with pytest.raises(P.PrismError) as e:
        P.HostFactor(A, P.PRECOND_ILDLT, tol=0.0)
    assert e.value.status == 3
    with pytest.raises(P.PrismError) as e:
        P.HostFactor(A, P.PRECOND_ILUT, tol=0.0, lfill=4)
    assert e.value.status == 3


@pytest.mark.parametrize("bad", ["unsorted", "range", "offsets"])
def test_bad_csr_rejected(bad):
    rp = np.array([0, 2, 4], np.uint32)
    ci = np.array([0, 1, 0, 1], np.uint32)
    v = np.array([2.0, -1.0, -1.0, 2.0])
    if bad == "unsorted":
        ci = np.array([1, 0, 0, 1], np.uint32)
    elif bad == "range":
        ci = np.array([0, 5, 0, 1], np.uint32)
    else:
        rp = np.array([0, 3, 2], np.uint32)
    with pytest.raises(P.PrismError) as e:
        P.HostFactor(P.CSRMatrix(rp, ci, v), P.PRECOND_IC, tol=0.0)
    assert e.value.status == 10


def test_single_row_and_diagonal():
    # ragged extremes: a 1x1 system and a diagonal matrix (no dependencies, one wavefront)
    A = P.CSRMatrix(np.array([0, 1], np.uint32), np.array([0], np.uint32), np.array([4.0]))
    F = P.HostFactor(A, P.PRECOND_IC, tol=0.0)
    rp, ci, v, _ = F.arrays(0)
    assert v.tolist() == [2.0] and F.info()["lower_levels"] == 1
    n = 17
    D = P.CSRMatrix(np.arange(n + 1, dtype=np.uint32), np.arange(n, dtype=np.uint32), np.arange(1.0, n + 1))
    F = P.HostFactor(D, P.PRECOND_ILUT, tol=0.0, lfill=3)
    assert F.info()["lower_levels"] == 1 and F.info()["upper_levels"] == 1
