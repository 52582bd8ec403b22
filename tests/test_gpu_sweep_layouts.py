"""Every device layout of the triangular sweep, forced in turn
(PRISM_SWEEP_KERNEL = global | slab | stream, read when a handle is created),
against the oracle and the reference's golden outputs: the triangular and
AMSED / GMSLR applies and FCG on them.  The setup-time tuner may pick any of
the three for a given sweep, so each must agree with the reference on its own.
Tolerances as in test_gpu_parity.py."""
from __future__ import annotations

import os

import numpy as np
import pytest

import prispack_b200 as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

KIND = {1: P.PRECOND_IC, 2: P.PRECOND_ILUT, 3: P.PRECOND_ILDLT}
KERNEL_ID = {"global": "level-order", "slab": "slab", "stream": "stream"}


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(params=["global", "slab", "stream"])
def layout(request):
    old = os.environ.get("PRISM_SWEEP_KERNEL")
    os.environ["PRISM_SWEEP_KERNEL"] = request.param
    yield request.param
    if old is None:
        del os.environ["PRISM_SWEEP_KERNEL"]
    else:
        os.environ["PRISM_SWEEP_KERNEL"] = old


def assert_layout(S, layout, sweeps):
    for sw in range(sweeps):
        info = S.sweep_info(sw)
        if info["n"]:
            assert info["kernel"] == KERNEL_ID[layout], (sw, info)


@pytest.mark.parametrize("name", ["lap2d_8", "lap3d_6", "conv2d_16", "lap2d_64"])
def test_triangular_apply(layout, name, manifest, load_golden):
    import torch
    g = load_golden(name)
    S = P.DeviceSystem(P.CSRMatrix(g["rowptr"], g["col"], g["val"]))
    for key, e in manifest[name]["precond"].items():
        if e.get("setup_rc") != 0:
            continue
        prec = P.PRISM_FP32 if key.endswith("fp32") else P.PRISM_FP64
        S.set_precond(KIND[e["kind"]], tol=e["tol"], lfill=e["lfill"], precision=prec)
        assert_layout(S, layout, 2)
        out = S.apply(g["probe"])
        assert rel_err(out, g[f"{key}.apply"]) < 1e-12, key
        # in-place apply through the device path (in == out)
        v = torch.tensor(g["probe"], device="cuda")
        assert S.lib.prism_apply_device(S.h, P._ptr(v), P._ptr(v)) == 0
        torch.cuda.synchronize()
        assert rel_err(v.cpu().numpy(), g[f"{key}.apply"]) < 1e-12, key


@pytest.mark.parametrize("prec", [P.PRISM_FP64, P.PRISM_FP32])
def test_fcg_ic_3d(layout, prec):
    A = P.CSRMatrix.laplacian(30, 26, 22)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3, precision=prec)
    assert_layout(S, layout, 2)
    b = np.random.default_rng(31).standard_normal(A.n)
    rp, ci, v, _ = S.precond_factor(0)
    pre = orc.Precond(1, A.n, (rp, ci, v))
    assert rel_err(S.apply(b), pre.apply(b)) < 1e-12
    x, st = S.solve(b, tol=1e-10, max_iter=1000)
    xo, ito, _, _ = orc.cg(A.rowptr, A.col, A.val, b, pre, tol=1e-10, maxit=1000)
    assert abs(st.num_iter - ito) <= 1 and st.converged
    if st.num_iter == ito:
        assert rel_err(x, xo) < 1e-10


@pytest.mark.parametrize("prec", [P.PRISM_FP32, P.PRISM_FP64])
def test_amsed_apply_and_fcg(layout, prec):
    A = P.CSRMatrix.laplacian(36, 32, 28)
    H = P.HostAmsed(A, levels=3, lanczos_steps=40, low_rank=16, lowrank_type=0, reorder=0, precision=prec)
    S = P.DeviceSystem(A)
    S.attach(H)
    assert_layout(S, layout, 6)
    b = np.random.default_rng(9).standard_normal(A.n)
    amsed = orc.Amsed(H)
    assert rel_err(S.apply(b), amsed.apply(b)) < 1e-12
    x, st = S.solve(b, tol=1e-10, max_iter=500)
    xo, ito, _, _ = orc.cg(A.rowptr, A.col, A.val, b, amsed.precond(), tol=1e-10, maxit=500)
    assert abs(st.num_iter - ito) <= 1 and st.converged
    if st.num_iter == ito:
        assert rel_err(x, xo) < 1e-10


def test_gmslr_apply(layout):
    A = P.CSRMatrix.laplacian(24, 24, 1)
    G = P.HostGmslr(A, levels=3, lanczos_steps=20, low_rank=8)
    S = P.DeviceSystem(A)
    S.attach(G)
    b = np.random.default_rng(10).standard_normal(A.n)
    assert rel_err(S.apply(b), orc.Amsed(G).apply(b)) < 1e-12


def test_single_sweeps_repeatable(layout):
    """Each sweep alone through the diagnostics entry point: prepare + sweep twice
    gives identical bits, and lower then upper equals the full apply."""
    import torch
    A = P.CSRMatrix.laplacian(40, 40, 40)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3, precision=P.PRISM_FP32)
    assert_layout(S, layout, 2)
    S.set_stream(torch.cuda.current_stream().cuda_stream)
    b = torch.tensor(np.random.default_rng(12).standard_normal(A.n), device="cuda")
    t = torch.empty_like(b)
    o1, o2 = torch.empty_like(b), torch.empty_like(b)
    S.sweep_device(0, b, t, 1)
    S.sweep_device(1, t, o1, 1)
    S.sweep_device(0, b, t, 1)
    S.sweep_device(1, t, o2, 1)
    torch.cuda.synchronize()
    assert torch.equal(o1, o2)
    assert rel_err(o1.cpu().numpy(), S.apply(b.cpu().numpy())) < 1e-13
