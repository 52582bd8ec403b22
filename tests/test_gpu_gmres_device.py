"""The device-side GMRES: each restart cycle as one CUDA graph whose Arnoldi loop
ends on the device, against the same kernels launched one by one and against
the oracle's GMRES (GMRES.cpp:122-221 restated, modified Gram-Schmidt).

The graph and the plain launches run the same kernels on the same grids, so
their results must be equal to the last bit; only the number of host waits
differs (one per restart cycle against one per Arnoldi step).  Against the
oracle, whose orthogonalisation is modified rather than classical Gram-Schmidt
applied twice, the solve-phase bar applies: iteration counts within +-1 and
solutions within 1e-10 relative when the counts agree."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

REL_SOL = 1e-10


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def convection_ilut():
    A = P.CSRMatrix.laplacian(24, 20, 16, 0.4, -0.25, 0.1)
    F = P.HostFactor(A, P.PRECOND_ILUT, tol=1e-2, lfill=20, precision=P.PRISM_FP32)
    S = P.DeviceSystem(A)
    S.attach(F)
    return A, F, S


@pytest.mark.parametrize("restart", [7, 30])
def test_cycle_graph_equals_plain_launches(restart):
    A, F, S = convection_ilut()
    b = np.random.default_rng(5).standard_normal(A.n)
    xg, sg = S.solve(b, solver=P.SOLVER_FGMRES, tol=1e-10, restart=restart)
    xs, ss = S.solve(b, solver=P.SOLVER_FGMRES, tol=1e-10, restart=restart, launch_mode=P.LAUNCH_STREAM)
    assert sg.graph_nodes > 0, "the restart cycle did not run as a graph"
    assert ss.graph_nodes == 0
    assert np.array_equal(xg, xs)
    assert (sg.num_iter, sg.converged, sg.final_error) == (ss.num_iter, ss.converged, ss.final_error)
    assert (sg.precond_applies, sg.spmv_count) == (ss.precond_applies, ss.spmv_count)
    cycles = sg.num_iter // restart + 1
    assert sg.host_syncs == cycles + 1           # one read per cycle and the final residual
    assert ss.host_syncs == cycles + 1 + sg.precond_applies  # and one per Arnoldi step
    assert sg.converged and sg.true_rel_residual < 1e-8


@pytest.mark.parametrize("restart", [7, 30])
def test_restarted_fgmres_vs_oracle(restart):
    A, F, S = convection_ilut()
    b = np.random.default_rng(11).standard_normal(A.n)
    x, st = S.solve(b, solver=P.SOLVER_FGMRES, tol=1e-10, restart=restart)
    f0, f1 = F.arrays(0), F.arrays(1)
    OP = orc.Precond(2, A.n, f0[:3], f1[:3], f1[3])
    xo, ito, erro, convo = orc.gmres(A.rowptr, A.col, A.val, b, OP, tol=1e-10, restart=restart)
    assert abs(st.num_iter - ito) <= 1 and bool(st.converged) == convo, (st.num_iter, ito)
    if st.num_iter == ito:
        assert rel_err(x, xo) < REL_SOL
    assert abs(st.final_error - erro) < 1e-12


def test_unpreconditioned_gmres_vs_oracle():
    A = P.CSRMatrix.laplacian(40, 30, 1, 0.3, 0.2, 0.0)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_NONE)
    b = np.random.default_rng(3).uniform(-1.0, 1.0, A.n)
    x, st = S.solve(b, solver=P.SOLVER_GMRES, tol=1e-8, restart=40)
    xo, ito, erro, convo = orc.gmres(A.rowptr, A.col, A.val, b, None, tol=1e-8, restart=40, flexible=False)
    assert abs(st.num_iter - ito) <= 1 and bool(st.converged) == convo, (st.num_iter, ito)
    if st.num_iter == ito:
        assert rel_err(x, xo) < REL_SOL


def test_lucky_breakdown_matches_oracle():
    """A diagonal matrix with three distinct values: the Krylov space is exhausted after
    three steps (GMRES.cpp:183-186 shortens the cycle there); both sides stop alike."""
    n = 300
    d = np.repeat([1.0, 2.0, 4.0], n // 3)
    rp = np.arange(n + 1, dtype=np.uint32)
    ci = np.arange(n, dtype=np.uint32)
    A = P.CSRMatrix(rp, ci, d)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_NONE)
    b = np.random.default_rng(8).uniform(0.5, 1.5, n)
    x, st = S.solve(b, solver=P.SOLVER_GMRES, tol=1e-12, restart=20)
    xo, ito, erro, convo = orc.gmres(rp, ci, d, b, None, tol=1e-12, restart=20, flexible=False)
    assert (st.num_iter, bool(st.converged)) == (ito, convo)
    assert rel_err(x, xo) < 1e-12
