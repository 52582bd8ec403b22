"""prism_residual_norms_noalloc, called through the C ABI, against the
existing entry points: the true relative residual that prism_solve_device
reports, and b - A x formed from prism_spmv_device.  Two calls in a row on the
same inputs must agree with those and with each other.  Collected last so that
it also runs after every other GPU test in the same process."""
from __future__ import annotations


import numpy as np
import pytest

import prispack_b200 as P

pytestmark = pytest.mark.gpu

K = 3  # right-hand sides in one call
PRISM_OK, PRISM_ERR_ARG = 0, 1  # prism_status values of include/prism_solve.h


def _noalloc(lib, dev, A_d, x, b, k, ld, norms, stream):
    rowptr, col, val = A_d
    return lib.prism_residual_norms_noalloc(dev, int(rowptr.numel() - 1), rowptr.data_ptr(), col.data_ptr(),
                                            val.data_ptr(), x.data_ptr(), b.data_ptr(), k, ld, norms.data_ptr(),
                                            stream)


def test_noalloc_residual_norms_match_existing_entry_points():
    import torch

    lib = P.load()
    dev = torch.cuda.current_device()
    A = P.CSRMatrix.laplacian(40, 40, 40, 0.0, 0.0, 0.0)   # n = 64000: every block strides over rows
    n = A.n
    A_d = (torch.from_numpy(A.rowptr.view(np.int32)).cuda(), torch.from_numpy(A.col.view(np.int32)).cuda(),
           torch.from_numpy(A.val).cuda())

    # existing path: an FCG + IC solve reports the true relative residual of its x
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3)
    rng = np.random.default_rng(11)
    b0 = torch.from_numpy(rng.uniform(-1, 1, n)).cuda()
    x0, st = S.solve(b0, tol=1e-8, max_iter=500)
    assert st.converged

    # k columns, column-major with leading dimension ld > n
    ld = n + 37
    X = torch.zeros(K * ld, dtype=torch.float64, device="cuda")
    B = torch.zeros(K * ld, dtype=torch.float64, device="cuda")
    X[:n] = x0
    B[:n] = b0
    for c in range(1, K):
        X[c * ld:c * ld + n] = torch.from_numpy(rng.standard_normal(n)).cuda()
        B[c * ld:c * ld + n] = torch.from_numpy(rng.standard_normal(n)).cuda()

    # existing path: y = A x per column through prism_spmv_device, norms on the host
    want = []
    for c in range(K):
        xc = X[c * ld:c * ld + n].contiguous()
        yc = S.spmv(xc)
        bc = B[c * ld:c * ld + n].cpu().numpy()
        r = bc - yc.cpu().numpy()
        want.append((np.linalg.norm(r), np.linalg.norm(bc)))

    stream = torch.cuda.current_stream().cuda_stream
    results = []
    for _ in range(2):  # two calls in a row
        norms = torch.full((2 * K,), float("nan"), dtype=torch.float64, device="cuda")
        rc = _noalloc(lib, dev, A_d, X, B, K, ld, norms, stream)
        assert rc == PRISM_OK, lib.prism_last_error()
        torch.cuda.synchronize()
        results.append(norms.cpu().numpy())

    for got in results:
        for c in range(K):
            # column 0 is a converged solution: its residual is a difference of nearly equal
            # vectors, so two SpMV summation orders differ by about eps * ||b||, not relative
            np.testing.assert_allclose(got[2 * c], want[c][0], rtol=1e-10, atol=1e-13 * want[c][1])
            np.testing.assert_allclose(got[2 * c + 1], want[c][1], rtol=1e-12)
        # column 0 against the solver's own true residual
        np.testing.assert_allclose(got[0] / got[1], st.true_rel_residual, rtol=1e-10, atol=1e-13)
    # same inputs, same fixed grid and reduction order: identical bits
    assert np.array_equal(results[0], results[1])

    # k = 1 ignores ld
    norms = torch.zeros(2, dtype=torch.float64, device="cuda")
    assert _noalloc(lib, dev, A_d, x0, b0, 1, 0, norms, stream) == PRISM_OK, lib.prism_last_error()
    torch.cuda.synchronize()
    np.testing.assert_allclose(norms.cpu().numpy(), results[0][:2], rtol=1e-12)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch

    lib = P.load()
    dev = torch.cuda.current_device()
    A = P.CSRMatrix.laplacian(8, 8, 1, 0.0, 0.0, 0.0)
    A_d = (torch.from_numpy(A.rowptr.view(np.int32)).cuda(), torch.from_numpy(A.col.view(np.int32)).cuda(),
           torch.from_numpy(A.val).cuda())
    X = torch.zeros(17 * A.n, dtype=torch.float64, device="cuda")
    norms = torch.zeros(34, dtype=torch.float64, device="cuda")
    rc = _noalloc(lib, dev, A_d, X, X, 17, A.n, norms, None)
    assert rc == PRISM_ERR_ARG
    assert b"16" in lib.prism_last_error()
    rc = _noalloc(lib, dev, A_d, X, X, 0, A.n, norms, None)
    assert rc == PRISM_ERR_ARG
    rc = _noalloc(lib, dev, A_d, X, X, 2, A.n - 1, norms, None)
    assert rc == PRISM_ERR_ARG and b"leading dimension" in lib.prism_last_error()


def test_noalloc_calls_take_no_device_memory():
    """After the first call on a device (which resolves the scratch address),
    a batch of calls leaves the device's free memory exactly where it was."""
    import torch

    lib = P.load()
    dev = torch.cuda.current_device()
    A = P.CSRMatrix.laplacian(32, 32, 32, 0.0, 0.0, 0.0)
    A_d = (torch.from_numpy(A.rowptr.view(np.int32)).cuda(), torch.from_numpy(A.col.view(np.int32)).cuda(),
           torch.from_numpy(A.val).cuda())
    rng = np.random.default_rng(12)
    X = torch.from_numpy(rng.standard_normal(4 * A.n)).cuda()
    B = torch.from_numpy(rng.standard_normal(4 * A.n)).cuda()
    norms = torch.zeros(8, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert _noalloc(lib, dev, A_d, X, B, 4, A.n, norms, stream) == PRISM_OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    for _ in range(20):
        assert _noalloc(lib, dev, A_d, X, B, 4, A.n, norms, stream) == PRISM_OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0


def test_noalloc_on_a_device_that_is_not_current():
    """With more than one GPU visible: a call naming another device runs there
    (its own scratch) and leaves the calling thread's current device as it was."""
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("needs two visible GPUs")
    lib = P.load()
    cur = torch.cuda.current_device()
    other = (cur + 1) % torch.cuda.device_count()
    A = P.CSRMatrix.laplacian(16, 16, 16, 0.0, 0.0, 0.0)
    with torch.cuda.device(other):
        A_d = (torch.from_numpy(A.rowptr.view(np.int32)).cuda(), torch.from_numpy(A.col.view(np.int32)).cuda(),
               torch.from_numpy(A.val).cuda())
        x = torch.from_numpy(np.random.default_rng(13).standard_normal(A.n)).cuda()
        b = torch.from_numpy(np.random.default_rng(14).standard_normal(A.n)).cuda()
        norms = torch.zeros(2, dtype=torch.float64, device="cuda")
    assert _noalloc(lib, other, A_d, x, b, 1, 0, norms, None) == PRISM_OK, lib.prism_last_error()
    assert torch.cuda.current_device() == cur
    torch.cuda.synchronize(other)
    r = b.cpu().numpy() - A.to_scipy() @ x.cpu().numpy()
    np.testing.assert_allclose(norms.cpu().numpy()[0], np.linalg.norm(r), rtol=1e-10)
