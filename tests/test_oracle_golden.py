"""The C oracle against the reference's own outputs (golden fixtures and, where
the reference build exists, the live reference).  CPU only."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle import oracle as orc
from oracle import ref

CASES = ["lap2d_8", "lap3d_6", "conv2d_16", "lap2d_64"]


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", CASES)
def test_laplacian_bit_exact(name, manifest, load_golden):
    g = load_golden(name)
    nx, ny, nz, ax, ay, az, sh = manifest[name]["grid"]
    rp, ci, v = orc.laplacian(nx, ny, nz, ax, ay, az, sh)
    assert np.array_equal(rp, g["rowptr"]) and np.array_equal(ci, g["col"]) and np.array_equal(v, g["val"])
    assert sha(rp, ci, v) == manifest[name]["A_sha"]


@pytest.mark.parametrize("name", CASES)
def test_spmv_matches_reference(name, load_golden):
    g = load_golden(name)
    y = orc.spmv(g["rowptr"], g["col"], g["val"], g["probe"])
    if ref.available():
        A = ref.RefCSR.from_arrays(g["rowptr"], g["col"], g["val"])
        assert np.array_equal(y, A.spmv(g["probe"]))
    # independent check with scipy
    import scipy.sparse as sp
    M = sp.csr_matrix((g["val"], g["col"], g["rowptr"]))
    np.testing.assert_allclose(y, M @ g["probe"], rtol=1e-14, atol=1e-14)


def _oracle_precond(g, key, kind):
    n = len(g["rowptr"]) - 1
    f0 = (g[f"{key}.f0_rowptr"], g[f"{key}.f0_col"], g[f"{key}.f0_val"])
    f1 = (g[f"{key}.f1_rowptr"], g[f"{key}.f1_col"], g[f"{key}.f1_val"]) if kind == 2 else None
    diag = g.get(f"{key}.diag")
    return orc.Precond(kind, n, f0, f1, diag)


def _full_keys(manifest, name):
    return [k for k, e in manifest[name]["precond"].items() if e.get("setup_rc") == 0]


@pytest.mark.parametrize("name", ["lap2d_8", "lap3d_6", "conv2d_16"])
def test_precond_apply_bit_exact(name, manifest, load_golden):
    """oracle MInvSolve on the reference's factor arrays == reference MInvSolve, bit for bit."""
    g = load_golden(name)
    for key in _full_keys(manifest, name):
        kind = manifest[name]["precond"][key]["kind"]
        P = _oracle_precond(g, key, kind)
        out = P.apply(g["probe"])
        assert np.array_equal(out, g[f"{key}.apply"]), key


@pytest.mark.parametrize("name", ["lap2d_8", "lap3d_6"])
def test_cg_matches_reference(name, manifest, load_golden):
    g = load_golden(name)
    for key in _full_keys(manifest, name):
        e = manifest[name]["precond"][key]
        if e["kind"] not in (1, 3):
            continue
        P = _oracle_precond(g, key, e["kind"])
        for flex in (True, False):
            tag = f"{key}.cg_{'flex' if flex else 'normal'}"
            x, it, err, conv = orc.cg(g["rowptr"], g["col"], g["val"], g["b"], P, tol=1e-8, maxit=1000,
                                      flexible=flex)
            assert it == e[tag]["iters"] and conv == e[tag]["conv"], tag
            assert err == e[tag]["err"], tag
            assert np.array_equal(x, g[f"{tag}.x"]), tag


@pytest.mark.parametrize("name", ["lap2d_8", "lap3d_6", "conv2d_16"])
def test_fgmres_matches_reference(name, manifest, load_golden):
    g = load_golden(name)
    for key in _full_keys(manifest, name):
        e = manifest[name]["precond"][key]
        P = _oracle_precond(g, key, e["kind"])
        tag = f"{key}.fgmres20"
        x, it, err, conv = orc.gmres(g["rowptr"], g["col"], g["val"], g["b"], P, tol=1e-8, restart=20,
                                     flexible=True)
        assert it == e[tag]["iters"] and conv == e[tag]["conv"], tag
        np.testing.assert_allclose(err, e[tag]["err"], rtol=1e-12)
        np.testing.assert_allclose(x, g[f"{tag}.x"], rtol=0, atol=1e-12 * np.abs(g[f"{tag}.x"]).max())


@pytest.mark.parametrize("name", CASES)
def test_unpreconditioned_solvers(name, manifest, load_golden):
    g = load_golden(name)
    m = manifest[name]
    if "none.cg" in m:
        x, it, err, conv = orc.cg(g["rowptr"], g["col"], g["val"], g["b"], None, tol=1e-8, maxit=1000)
        assert it == m["none.cg"]["iters"]
        np.testing.assert_allclose(x, g["none.cg.x"], rtol=0, atol=1e-12 * np.abs(x).max())
    x, it, err, conv = orc.gmres(g["rowptr"], g["col"], g["val"], g["b"], None, tol=1e-8, restart=30, flexible=False)
    assert it == m["none.gmres30"]["iters"]
    np.testing.assert_allclose(x, g["none.gmres30.x"], rtol=0, atol=1e-12 * np.abs(x).max())


@pytest.mark.skipif(not ref.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("grid", [(12, 9, 7), (40, 40, 1), (5, 1, 1)])
def test_oracle_vs_live_reference(grid):
    """Seeds and shapes beyond the fixtures, against the reference build itself."""
    nx, ny, nz = grid
    A = ref.RefCSR.laplacian(nx, ny, nz, 0.1, 0.0, -0.05, 0.0)
    rp, ci, v = A.arrays()
    assert all(np.array_equal(a, b) for a, b in zip((rp, ci, v), orc.laplacian(nx, ny, nz, 0.1, 0.0, -0.05, 0.0)))
    b = np.random.default_rng(7).uniform(-1, 1, len(rp) - 1)
    P = ref.RefPrecond(A, ref.KIND_ILUT, False, 1e-3, 10)
    assert P.setup() == 0
    f0, f1 = P.factor(0), P.factor(1)
    OP = orc.Precond(2, len(rp) - 1, f0[:3], f1[:3], f1[3])
    assert np.array_equal(OP.apply(b), P.apply(b))
    xr, itr, _, _ = ref.gmres_solve(A, P, b, tol=1e-9, restart=15)
    xo, ito, _, _ = orc.gmres(rp, ci, v, b, OP, tol=1e-9, restart=15)
    assert itr == ito
    np.testing.assert_allclose(xo, xr, rtol=0, atol=1e-11 * np.abs(xr).max())
