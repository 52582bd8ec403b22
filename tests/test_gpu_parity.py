"""GPU parity: the sm_100a kernels, called through the C ABI, against the oracle
and the reference's golden outputs.  Tolerances: FP64 vectors with FP64 or FP32
factor values; reductions on the GPU sum in a different order than the serial
reference, so vector results agree to ~1e-13 relative, and solver results
satisfy the solve-phase bar: iteration counts within +-1 and solutions within
1e-10 relative when the iteration counts agree."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

KIND = {1: P.PRECOND_IC, 2: P.PRECOND_ILUT, 3: P.PRECOND_ILDLT}
REL_VEC = 1e-12       # apply / SpMV, relative to max |value|
REL_SOL = 1e-10       # solution agreement at equal iteration counts


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def system(g):
    return P.DeviceSystem(P.CSRMatrix(g["rowptr"], g["col"], g["val"]))


@pytest.mark.parametrize("name", ["lap2d_8", "lap3d_6", "conv2d_16", "lap2d_64"])
def test_spmv(name, load_golden):
    g = load_golden(name)
    S = system(g)
    y = S.spmv(g["probe"])
    assert rel_err(y, orc.spmv(g["rowptr"], g["col"], g["val"], g["probe"])) < 1e-14


@pytest.mark.parametrize("name", ["lap2d_8", "lap3d_6", "conv2d_16", "lap2d_64"])
def test_precond_apply(name, manifest, load_golden):
    g = load_golden(name)
    S = system(g)
    for key, e in manifest[name]["precond"].items():
        if e.get("setup_rc") != 0:
            continue
        prec = P.PRISM_FP32 if key.endswith("fp32") else P.PRISM_FP64
        S.set_precond(KIND[e["kind"]], tol=e["tol"], lfill=e["lfill"], precision=prec)
        assert S.precond_nnz() == e["mnnz"]
        out = S.apply(g["probe"])
        assert rel_err(out, g[f"{key}.apply"]) < REL_VEC, key


@pytest.mark.parametrize("name", ["lap2d_8", "lap3d_6", "lap2d_64"])
@pytest.mark.parametrize("flex", [True, False])
def test_cg_against_reference(name, flex, manifest, load_golden):
    g = load_golden(name)
    S = system(g)
    for key, e in manifest[name]["precond"].items():
        if e.get("setup_rc") != 0 or e["kind"] not in (1, 3):
            continue
        prec = P.PRISM_FP32 if key.endswith("fp32") else P.PRISM_FP64
        S.set_precond(KIND[e["kind"]], tol=e["tol"], precision=prec)
        tag = f"{key}.cg_{'flex' if flex else 'normal'}"
        x, st = S.solve(g["b"], solver=P.SOLVER_FCG if flex else P.SOLVER_CG, tol=1e-8, max_iter=1000)
        ref_it = e[tag]["iters"]
        assert abs(st.num_iter - ref_it) <= 1, (tag, st.num_iter, ref_it)
        assert bool(st.converged) == e[tag]["conv"]
        assert st.true_rel_residual < 1e-8 * 1.5, tag
        if st.num_iter == ref_it:
            assert rel_err(x, g[f"{tag}.x"]) < REL_SOL, tag


def test_config1_fcg_ict(load_golden, manifest):
    """2D Poisson 64x64, FCG + ICT(1e-3), b = U[-1,1], tol 1e-8, maxit 1000 (the reference's CPU case)."""
    g = load_golden("lap2d_64")
    S = system(g)
    S.set_precond(P.PRECOND_IC, tol=1e-3)
    x, st = S.solve(g["b"], tol=1e-8, max_iter=1000)
    e = manifest["lap2d_64"]["precond"]["ic_1e-3_fp64"]["ic_1e-3_fp64.cg_flex"]
    assert st.num_iter == e["iters"] == 15
    assert rel_err(x, g["ic_1e-3_fp64.cg_flex.x"]) < REL_SOL
    assert abs(st.final_error - e["err"]) < 1e-12


@pytest.mark.parametrize("grid,prec", [((32, 32, 32), P.PRISM_FP64), ((32, 32, 32), P.PRISM_FP32),
                                       ((48, 40, 20), P.PRISM_FP64)])
def test_fcg_3d_against_oracle(grid, prec):
    """Larger 3D problems: product factor -> GPU FCG vs the oracle FCG on the same factor."""
    A = P.CSRMatrix.laplacian(*grid)
    F = P.HostFactor(A, P.PRECOND_IC, tol=1e-3, precision=prec)
    S = P.DeviceSystem(A)
    S.attach(F)
    b = np.random.default_rng(3).standard_normal(A.n)
    x, st = S.solve(b, tol=1e-10, max_iter=1000)
    rp, ci, v, _ = F.arrays(0)
    OP = orc.Precond(1, A.n, (rp, ci, v))
    xo, ito, erro, convo = orc.cg(A.rowptr, A.col, A.val, b, OP, tol=1e-10, maxit=1000)
    assert abs(st.num_iter - ito) <= 1
    assert st.true_rel_residual < 2e-10
    if st.num_iter == ito:
        assert rel_err(x, xo) < REL_SOL


def test_device_pointer_path_matches_host_path():
    import torch
    A = P.CSRMatrix.laplacian(20, 20, 20)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_ILDLT, tol=1e-3)
    b = np.random.default_rng(5).uniform(-1, 1, A.n)
    xh, sth = S.solve(b, tol=1e-9)
    bd = torch.tensor(b, device="cuda")
    xd, std = S.solve(bd, tol=1e-9)
    assert sth.num_iter == std.num_iter
    assert np.array_equal(xh, xd.cpu().numpy())   # same kernels, same order: bitwise
    yd = S.apply(bd)
    assert np.array_equal(yd.cpu().numpy(), S.apply(b))


def test_repeatable_bitwise():
    A = P.CSRMatrix.laplacian(30, 30, 30)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3, precision=P.PRISM_FP32)
    b = np.random.default_rng(9).standard_normal(A.n)
    x1, s1 = S.solve(b, tol=1e-10)
    x2, s2 = S.solve(b, tol=1e-10)
    assert s1.num_iter == s2.num_iter and np.array_equal(x1, x2)


def test_launch_counter_moves():
    before = P.kernel_launch_count()
    A = P.CSRMatrix.laplacian(8, 8, 1)
    S = P.DeviceSystem(A)
    S.spmv(np.ones(A.n))
    assert P.kernel_launch_count() > before


def test_bounded_wait_times_out_and_context_survives():
    """A sweep row waits for a value nothing produces: the wait runs out (50 ms),
    the kernel reports PRISM_ERR_TIMEOUT, and the context keeps working."""
    import time
    t = time.time()
    assert P.selftest_wait_timeout(0, 50_000_000) == 6
    assert time.time() - t < 10
    A = P.CSRMatrix.laplacian(8, 8, 1)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3)
    x, st = S.solve(np.ones(A.n), tol=1e-8)
    assert st.converged


@pytest.mark.parametrize("name", ["lap2d_8", "lap3d_6", "conv2d_16", "lap2d_64"])
def test_fgmres_against_reference(name, manifest, load_golden):
    """FlexibleGMRES with setRestart(true, 20) against the reference's outputs."""
    g = load_golden(name)
    S = system(g)
    for key, e in manifest[name]["precond"].items():
        if e.get("setup_rc") != 0:
            continue
        prec = P.PRISM_FP32 if key.endswith("fp32") else P.PRISM_FP64
        S.set_precond(KIND[e["kind"]], tol=e["tol"], lfill=e["lfill"], precision=prec)
        tag = f"{key}.fgmres20"
        x, st = S.solve(g["b"], solver=P.SOLVER_FGMRES, tol=1e-8, restart=20)
        ref = e[tag]
        assert abs(st.num_iter - ref["iters"]) <= 1, (tag, st.num_iter, ref["iters"])
        assert bool(st.converged) == ref["conv"]
        if st.num_iter == ref["iters"]:
            assert rel_err(x, g[f"{tag}.x"]) < REL_SOL, tag


@pytest.mark.parametrize("name", ["lap2d_8", "lap3d_6", "conv2d_16", "lap2d_64"])
def test_gmres_unpreconditioned_against_reference(name, manifest, load_golden):
    g = load_golden(name)
    S = system(g)
    S.set_precond(P.PRECOND_NONE)
    x, st = S.solve(g["b"], solver=P.SOLVER_GMRES, tol=1e-8, restart=30)
    ref = manifest[name]["none.gmres30"]
    assert abs(st.num_iter - ref["iters"]) <= 1, (st.num_iter, ref["iters"])
    if st.num_iter == ref["iters"]:
        assert rel_err(x, g["none.gmres30.x"]) < REL_SOL


def test_fgmres_convection_3d_against_oracle():
    """Nonsymmetric 3D problem beyond the fixtures: ILUT(20, 1e-2) + FGMRES(30), GPU vs oracle."""
    A = P.CSRMatrix.laplacian(24, 20, 16, 0.4, -0.25, 0.1)
    F = P.HostFactor(A, P.PRECOND_ILUT, tol=1e-2, lfill=20, precision=P.PRISM_FP32)
    S = P.DeviceSystem(A)
    S.attach(F)
    b = np.random.default_rng(11).standard_normal(A.n)
    x, st = S.solve(b, solver=P.SOLVER_FGMRES, tol=1e-10, restart=30)
    f0, f1 = F.arrays(0), F.arrays(1)
    OP = orc.Precond(2, A.n, f0[:3], f1[:3], f1[3])
    xo, ito, erro, convo = orc.gmres(A.rowptr, A.col, A.val, b, OP, tol=1e-10, restart=30)
    assert abs(st.num_iter - ito) <= 1 and st.converged == convo
    if st.num_iter == ito:
        assert rel_err(x, xo) < REL_SOL
    assert abs(st.final_error - erro) < 1e-12
