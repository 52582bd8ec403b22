"""Parity with the reference's own solver at the benchmark configurations'
sizes (the compiled reference, oracle/_ref, built from its sources by
oracle/Makefile; a CPU build that travels with the repository).

* 2D Poisson 64^2, FCG + ICT(1e-3), tol 1e-8 (the reference's own CPU case):
  CG<double> + IncompleteCholesky<double, double> (CG.cpp:34-83).
* 3D Poisson 64^3, FCG + AMSED/MSLR (3 levels, rank <= 32), tol 1e-10, FP64
  factors: CG<double> + AMSEDPrecondition<double, double>
  (AMSEDPrecondition.cpp:1976-2087).
* 3D convection-diffusion 40^3 (the nonsymmetric configuration on a smaller
  grid), FGMRES(50) + GMSLR (4 levels, rank 24), tol 1e-10, FP64 factors:
  GMRES<double> + GMSLRPrecondition<double, double> (GMRES.cpp:122-221).

Bar: iteration counts within 1 and, when they agree, solutions within 1e-10
relative (the solver's own forward-error report, stats.forward_error, against
the reference's x).  The single-precision apply (PRISM_FP32_APPLY) reaches the
same tolerance; its solution is compared with the reference's FP64 one within
1e-7, the spread that two solutions with relative residual 1e-10 may have on
these condition numbers."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P
from oracle import ref

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref.available(), reason="reference build (oracle/_ref) absent")]

AMSED = dict(levels=3, lanczos_steps=64, low_rank=32, eig_bound=0.8, lowrank_type=0, lanczos_type=0, reorder=0)


def test_config1_64sq_fcg_ict_against_reference():
    A = P.CSRMatrix.laplacian(64, 64, 1)
    b = np.random.default_rng(2024).uniform(-1.0, 1.0, A.n)
    RA = ref.RefCSR.laplacian(64, 64, 1)
    RP = ref.RefPrecond(RA, ref.KIND_IC, False, 1e-3)
    RP.setup()
    xr, itr, _, conv = ref.cg_solve(RA, RP, b, tol=1e-8, maxit=1000, flexible=True)
    assert conv
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3)
    x, st = S.solve(b, tol=1e-8, max_iter=1000, x_ref=xr)
    assert st.converged and abs(st.num_iter - itr) <= 1
    assert st.forward_error == pytest.approx(np.linalg.norm(x - xr) / np.linalg.norm(xr), rel=1e-6, abs=1e-16)
    if st.num_iter == itr:
        assert st.forward_error <= 1e-10


def test_64cube_fcg_amsed_fp64_against_reference():
    g = 64
    A = P.CSRMatrix.laplacian(g, g, g)
    b = np.random.default_rng(2024).standard_normal(A.n)
    RA = ref.RefCSR.laplacian(g, g, g)
    a = AMSED
    RP = ref.RefAmsed(RA, a["levels"], a["lanczos_steps"], a["low_rank"], a["eig_bound"], a["reorder"],
                      a["lowrank_type"], a["lanczos_type"], False)
    RP.setup()
    xr, itr, _, conv = ref.cg_solve(RA, RP, b, tol=1e-10, maxit=1000, flexible=True)
    assert conv
    S = P.DeviceSystem(A)
    S.set_amsed(precision=P.PRISM_FP64, **AMSED)
    x, st = S.solve(b, tol=1e-10, max_iter=1000, x_ref=xr)
    assert st.converged and abs(st.num_iter - itr) <= 1, (st.num_iter, itr)
    if st.num_iter == itr:
        assert st.forward_error <= 1e-10, st.forward_error
    # the mixed solve of the benchmark, against the same FP64 reference solution
    S.set_amsed(precision=P.PRISM_FP32_APPLY, **AMSED)
    _, st32 = S.solve(b, tol=1e-10, max_iter=1000, x_ref=xr)
    assert st32.converged and st32.true_rel_residual <= 1e-10
    assert st32.forward_error <= 1e-7, st32.forward_error


def test_40cube_convdiff_fgmres_gmslr_fp64_against_reference():
    g, pe = 40, 50.0
    A = P.CSRMatrix.convection_diffusion(g, g, g, pe, 0.5 * pe, 0.25 * pe)
    b = np.random.default_rng(2024).standard_normal(A.n)
    RA = ref.RefCSR.from_arrays(A.rowptr, A.col, A.val)
    RG = ref.RefGmslr(RA, 4, 20, 24, low_precision=False)
    RG.setup()
    xr, itr, _, conv = ref.gmres_solve(RA, RG, b, tol=1e-10, restart=50, flexible=True)
    assert conv
    G = P.HostGmslr(A, levels=4, low_rank=24, precision=P.PRISM_FP64)
    S = P.DeviceSystem(A)
    S.attach(G)
    x, st = S.solve(b, solver=P.SOLVER_FGMRES, tol=1e-10, max_iter=1000, restart=50, x_ref=xr)
    assert st.converged and abs(st.num_iter - itr) <= 1, (st.num_iter, itr)
    if st.num_iter == itr:
        assert st.forward_error <= 1e-10, st.forward_error
