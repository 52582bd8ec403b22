"""Matrix Market ingestion (prism_mtx_read) against the reference's own reader,
HOST::ReadMtxTools<double>::loadMatrix (source/utils/TestTools/ReadMtxTools.cpp):
the golden arrays in tests/golden/mtx_cases.npz were made by the compiled
reference from the fixture files in tests/golden/mtx/ (make_golden.py, section
mtx) -- general files with explicit zeros, duplicates, comments and unsorted
entries, symmetric and skew-symmetric files (expanded to the full matrix),
complex and hermitian files (real and imaginary parts), a rectangular one.
The CSR arrays must be identical."""
from __future__ import annotations

import os

import numpy as np
import pytest

import prispack_b200 as P
from oracle import ref

GOLD = os.path.join(os.path.dirname(__file__), "golden")
CASES = [("general", 0), ("symmetric", 0), ("skew", 0), ("complex", 0), ("complex", 1), ("hermitian", 0),
         ("hermitian", 1), ("rect", 0)]


@pytest.fixture(scope="module")
def gold():
    with np.load(os.path.join(GOLD, "mtx_cases.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name,part", CASES)
def test_reader_matches_reference_reader(name, part, gold):
    A = P.CSRMatrix.from_mtx(os.path.join(GOLD, "mtx", f"{name}.mtx"), part=part)
    key = f"{name}.{part}"
    assert np.array_equal(A.rowptr, gold[key + ".rowptr"])
    assert np.array_equal(A.col, gold[key + ".col"])
    assert np.array_equal(A.val.view(np.uint64), gold[key + ".val"].view(np.uint64))


@pytest.mark.skipif(not ref.available(), reason="reference checker build absent")
@pytest.mark.parametrize("name,part", CASES)
def test_reader_matches_reference_reader_live(name, part):
    path = os.path.join(GOLD, "mtx", f"{name}.mtx")
    rp, ci, v = ref.RefCSR.from_mtx(path, part).arrays()
    A = P.CSRMatrix.from_mtx(path, part=part)
    assert np.array_equal(A.rowptr, rp) and np.array_equal(A.col, ci) and np.array_equal(A.val, v)


def test_symmetric_file_expands_to_the_full_matrix(tmp_path):
    A = P.CSRMatrix.laplacian(6, 5, 4, 0.0, 0.0, 0.0)
    A.write_mtx(str(tmp_path / "s.mtx"), symmetric=True)
    B = P.CSRMatrix.from_mtx(str(tmp_path / "s.mtx"))
    assert np.array_equal(A.rowptr, B.rowptr) and np.array_equal(A.col, B.col) and np.array_equal(A.val, B.val)


def test_right_hand_side_array():
    X = P.read_mtx_dense(os.path.join(GOLD, "mtx", "rhs.mtx"))
    vals = [float(t) for t in open(os.path.join(GOLD, "mtx", "rhs.mtx")).read().split("\n")[3:] if t.strip()]
    assert X.shape == (2, 30)
    assert np.array_equal(X.ravel(), np.array(vals))


@pytest.mark.parametrize("text,why", [
    ("%%MatrixMarket matrix coordinate pattern general\n2 2 1\n1 1\n", "not supported"),
    ("%%MatrixMarket matrix coordinate integer general\n2 2 1\n1 1 3\n", "not supported"),
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", "coordinate"),
    ("% no banner\n2 2 1\n1 1 1.0\n", "banner"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n", "out of range"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1.0\n", "entries"),
])
def test_reader_refuses_what_it_cannot_read(tmp_path, text, why):
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    with pytest.raises(P.PrismError, match=why):
        P.CSRMatrix.from_mtx(str(p))


@pytest.mark.gpu
def test_solve_a_matrix_read_from_a_file(tmp_path):
    """End to end: a file written from the 3D Poisson matrix, read back and solved
    with FCG + IC on the device to 1e-10."""
    A0 = P.CSRMatrix.laplacian(20, 20, 20, 0.0, 0.0, 0.0)
    A0.write_mtx(str(tmp_path / "p.mtx"), symmetric=True)
    A = P.CSRMatrix.from_mtx(str(tmp_path / "p.mtx"))
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3)
    b = np.random.default_rng(3).standard_normal(A.n)
    x, st = S.solve(b, tol=1e-10, max_iter=500)
    assert st.converged and st.true_rel_residual <= 1e-10
