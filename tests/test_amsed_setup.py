"""AMSED / MSLR host setup and the oracle's AMSED apply against the reference
(golden fixtures from the reference build; live reference where present).  CPU only."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

import prispack_b200 as P
from oracle import oracle as orc
from oracle import ref

CASES = ["amsed_12c_mslr", "amsed_16c_defl32", "amsed_40sq_l4", "amsed_14x11x9_restart", "amsed_20c_defl_restart32"]


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def build(entry):
    A = P.CSRMatrix.laplacian(*entry["grid"])
    H = P.HostAmsed(A, levels=entry["levels"], lanczos_steps=entry["lanczos_steps"], low_rank=entry["low_rank"],
                    lowrank_type=entry["lowrank_type"], lanczos_type=entry.get("lanczos_type", 0), seed=entry["seed"],
                    precision=P.PRISM_FP32 if entry["fp32"] else P.PRISM_FP64)
    return A, H


@pytest.mark.parametrize("name", CASES)
def test_hid_and_factors_bit_exact(name, manifest):
    e = manifest["_amsed"][name]
    A, H = build(e)
    inf = H.info()
    assert inf["nlev"] == e["nlev"]
    assert inf["lev_ptr"].tolist() == e["lev_ptr"] and inf["ncomps"].tolist() == e["ncomps"]
    assert sha(H.perm()) == e["perm_sha"]
    assert inf["mnnz"] == e["mnnz"] and inf["ranks"].tolist() == e["ranks"]
    for lv in range(e["nlev"]):
        blk = e["blocks"][str(lv)]
        assert H.dom_ptr(lv).tolist() == blk["dom_ptr"]
        for b, digest in enumerate(blk["sha"]):
            rp, ci, v, d = H.block(lv, b)
            got = sha(rp, ci, v) + ("" if lv == e["nlev"] - 1 else sha(d))
            assert got == digest, (lv, b)
        if "H" in blk:
            # low-rank terms come from the Lanczos process and an eigen-decomposition: rounding-level agreement
            np.testing.assert_allclose(sorted(H.lowrank(lv)[1]), blk["H"], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("name", CASES)
def test_oracle_amsed_apply_and_fcg(name, manifest, load_golden):
    e = manifest["_amsed"][name]
    g = load_golden(name)
    A, H = build(e)
    O = orc.Amsed(H)
    out = O.apply(g["probe"])
    assert np.abs(out - g["apply"]).max() / np.abs(g["apply"]).max() < 1e-11
    x, it, err, conv = orc.cg(A.rowptr, A.col, A.val, g["b"], O.precond(), tol=1e-10, maxit=500)
    assert it == e["cg"]["iters"] and conv
    assert np.abs(x - g["cg.x"]).max() / np.abs(g["cg.x"]).max() < 1e-10


@pytest.mark.skipif(not ref.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("grid", [(9, 7, 5), (30, 1, 1), (17, 13, 1), (6, 6, 6)])
def test_rcm_matches_vendored_genrcm(grid):
    """The restated genrcm (used on every HID sub-domain) against the vendored one.
    A single-level AMSED orders the whole connected matrix with RCM."""
    A = P.CSRMatrix.laplacian(*grid)
    H = P.HostAmsed(A, levels=1, lanczos_steps=4, low_rank=2)
    assert np.array_equal(H.perm(), ref.rcm(A.rowptr, A.col))


def test_disconnected_graph_components():
    """Two decoupled 2D grids: the HID recursion sees two components, each bisected."""
    import scipy.sparse as sp
    A1 = P.CSRMatrix.laplacian(10, 10, 1).to_scipy()
    M = sp.block_diag([A1, A1]).tocsr()
    M.sort_indices()
    A = P.CSRMatrix(M.indptr, M.indices, M.data)
    H = P.HostAmsed(A, levels=2, lanczos_steps=10, low_rank=4)
    inf = H.info()
    assert inf["nlev"] == 2 and inf["ncomps"][1] == 2
    assert sorted(H.perm().tolist()) == list(range(A.n))


@pytest.mark.skipif(not ref.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("grid,levels,lt,low", [((14, 11, 9), 3, 0, False), ((20, 20, 20), 3, 1, True),
                                                 ((64, 48, 1), 5, 0, False)])
def test_live_reference_amsed(grid, levels, lt, low):
    A = P.CSRMatrix.laplacian(*grid)
    H = P.HostAmsed(A, levels=levels, lanczos_steps=30, low_rank=16, lowrank_type=lt,
                    precision=P.PRISM_FP32 if low else P.PRISM_FP64)
    R = ref.RefAmsed(ref.RefCSR.laplacian(*grid), levels, 30, 16, 0.8, 2, lt, 0, low)
    assert R.setup() == 0
    ri, pi = R.info(), H.info()
    assert np.array_equal(ri["lev_ptr"], pi["lev_ptr"]) and np.array_equal(R.perm(), H.perm())
    assert np.array_equal(ri["ranks"], pi["ranks"]) and ri["mnnz"] == pi["mnnz"]
    for lv in range(ri["nlev"]):
        nb = 1 if lv == ri["nlev"] - 1 else int(ri["ncomps"][lv])
        for b in range(nb):
            a, c = R.block(lv, b), H.block(lv, b)
            assert all(np.array_equal(x, y) for x, y in zip(a[:3], c[:3]))
    v = np.random.default_rng(4).standard_normal(A.n)
    ra = R.apply(v)
    # W comes from each side's own tridiagonal eigen-solver (LAPACK dstevx vs the product's QL
    # eigenvalues with inverse-iteration eigenvectors): within clusters of close Ritz values the
    # eigenvectors may rotate, so the apply agrees to the accuracy of the Ritz pairs rather than
    # to rounding.
    assert np.abs(orc.Amsed(H).apply(v) - ra).max() / np.abs(ra).max() < 1e-8


def random_spd(nx, ny, nz, seed):
    """A 7-point pattern with symmetric random off-diagonal weights: no symmetric degeneracy."""
    A = P.CSRMatrix.laplacian(nx, ny, nz)
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    v = A.val.copy()
    off = rows != A.col
    key = np.minimum(rows, A.col).astype(np.int64) * A.n + np.maximum(rows, A.col)
    uniq, inv = np.unique(key, return_inverse=True)
    v[off] *= rng.uniform(0.3, 1.0, len(uniq))[inv][off]
    return P.CSRMatrix(A.rowptr, A.col, v)


@pytest.mark.skipif(not ref.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("grid,levels,lt,low,rand", [((14, 11, 9), 3, 0, False, True), ((30, 30, 1), 3, 1, False, True),
                                                      ((20, 20, 20), 3, 1, True, False),
                                                      ((64, 48, 1), 5, 0, False, True),
                                                      ((64, 48, 1), 5, 0, False, False)])
def test_live_reference_restarted_lanczos(grid, levels, lt, low, rand):
    """UseRestartLanczos (AMSEDPrecondition.cpp:1010-1274) against the reference build.

    The reference applies each Givens rotation of its restart to the Ritz vectors as they
    were before any rotation (transposedGivensApplied2Columns reads the other buffer), so its
    low-rank W depends on the last components of converged Ritz vectors (1e-20 and below):
    the product computes those by inverse iteration, as dstevx does, and the low-rank terms,
    level by level, and the apply agree to rounding."""
    A = random_spd(*grid, 3) if rand else P.CSRMatrix.laplacian(*grid)
    H = P.HostAmsed(A, levels=levels, lanczos_steps=30, low_rank=16, lowrank_type=lt, lanczos_type=1,
                    precision=P.PRISM_FP32 if low else P.PRISM_FP64)
    R = ref.RefAmsed(ref.RefCSR.from_arrays(A.rowptr, A.col, A.val), levels, 30, 16, 0.8, 2, lt, 1, low)
    assert R.setup() == 0
    ri, pi = R.info(), H.info()
    assert np.array_equal(ri["ranks"], pi["ranks"]) and ri["mnnz"] == pi["mnnz"]
    assert ri["ranks"].max() > 0
    for lv in range(ri["nlev"] - 1):
        (rw, rh), (hw, hh) = R.lowrank(lv), H.lowrank(lv)
        if len(rh) == 0:
            continue
        np.testing.assert_allclose(np.sort(hh), np.sort(rh), rtol=1e-12, atol=1e-14 * np.abs(rh).max())
        Mr, Mh = (rw * rh) @ rw.T, (hw * hh) @ hw.T
        assert np.abs(Mh - Mr).max() <= 1e-11 * np.abs(Mr).max(), lv
    v = np.random.default_rng(4).standard_normal(A.n)
    ra = R.apply(v)
    assert np.abs(orc.Amsed(H).apply(v) - ra).max() <= 1e-11 * np.abs(ra).max()
