"""Adjoint solve (prism_adjoint_solve*) and the differentiable solve built on it
(prispack_b200.autograd), on the variable-coefficient diffusion problem:
against a dense FP64 reference gradient (torch autograd through a dense
solve, CPU) and against central finite differences with h = 1e-6."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P
from prispack_b200.autograd import DiffusionPattern, SolveSpec, gaussian_random_field, solve

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_adjoint_matches_dense_transpose_solve():
    D = DiffusionPattern(9, 7, 6)
    kappa = np.exp(gaussian_random_field(D.shape, 1.0, 3.0, seed=1))
    A = D.matrix(kappa)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_IC, tol=1e-3)
    rng = np.random.default_rng(2)
    b, g = rng.standard_normal(A.n), rng.standard_normal(A.n)
    x, st = S.solve(b, tol=1e-13, max_iter=2000)
    lam, gv, st2 = S.adjoint(g, x, tol=1e-13, max_iter=2000)
    Ad = A.to_scipy().toarray()
    lam_ref = np.linalg.solve(Ad.T, g)
    x_ref = np.linalg.solve(Ad, b)
    assert st2.converged and rel_err(lam, lam_ref) < 1e-10
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr.astype(np.int64)))
    assert rel_err(gv, -lam_ref[rows] * x_ref[A.col]) < 1e-10


def test_autograd_kappa_and_b_vs_dense_reference():
    import torch
    D = DiffusionPattern(7, 6, 5)
    g = gaussian_random_field(D.shape, 1.0, 2.0, seed=3)
    rng = np.random.default_rng(4)
    b0, xs = rng.standard_normal(D.n), rng.standard_normal(D.n)
    S = P.DeviceSystem(D.matrix(np.exp(g)))
    # device: the library's solve and adjoint
    kap = torch.tensor(np.exp(g), dtype=torch.float64, device="cuda", requires_grad=True)
    b = torch.tensor(b0, device="cuda", requires_grad=True)
    x = solve(S, D.values(kap), b, SolveSpec(tol=1e-13))
    loss = ((x - torch.tensor(xs, device="cuda")) ** 2).sum()
    loss.backward()
    # dense FP64 reference on the host: autograd through torch.linalg.solve
    kc = torch.tensor(np.exp(g), dtype=torch.float64, requires_grad=True)
    bc = torch.tensor(b0, requires_grad=True)
    v = D.values(kc)
    rp = torch.as_tensor(D.A0.rowptr.astype(np.int64))
    rows = torch.repeat_interleave(torch.arange(D.n), rp[1:] - rp[:-1])
    Ad = torch.zeros(D.n, D.n, dtype=torch.float64).index_put((rows, torch.as_tensor(D.A0.col.astype(np.int64))), v)
    xr = torch.linalg.solve(Ad, bc)
    lr = ((xr - torch.tensor(xs)) ** 2).sum()
    lr.backward()
    assert abs(loss.item() - lr.item()) / lr.item() < 1e-10
    assert rel_err(kap.grad.cpu().numpy(), kc.grad.numpy()) < 1e-8
    assert rel_err(b.grad.cpu().numpy(), bc.grad.numpy()) < 1e-8


def _fd_gradient(S, D, kappa, b, xs, m, h, tol):
    """Central difference (L(k + h e_m) - L(k - h e_m)) / (2h), L = ||x - xs||^2,
    evaluated without cancellation: with A- x- = b and A+ x+ = b,
    x+ - x- = -A+^{-1} (A+ - A-) x-, so L+ - L- = d . (2 x- + d - 2 xs)."""
    import torch
    kp, km = kappa.copy(), kappa.copy()
    kp[m] += h
    km[m] -= h
    vp = D.values(torch.from_numpy(kp)).numpy()
    vm = D.values(torch.from_numpy(km)).numpy()
    S.update_values(vm)
    xm, st = S.solve(b, tol=tol, max_iter=5000)
    dv = vp - vm
    rows = np.repeat(np.arange(D.n), np.diff(D.A0.rowptr.astype(np.int64)))
    r = np.zeros(D.n)
    np.add.at(r, rows, dv * xm[D.A0.col])
    S.update_values(vp)
    d, st2 = S.solve(-r, tol=tol, max_iter=5000)
    assert st.converged and st2.converged
    return float(d @ (2 * xm + d - 2 * xs)) / (2 * h)


@pytest.mark.parametrize("grid,ncoef", [((16, 16, 16), 16), ((64, 64, 64), 64)])
def test_autograd_vs_central_differences(grid, ncoef):
    """Variable-coefficient diffusion, kappa = exp(g) with g a Gaussian random
    field (sigma 1, correlation length 8 cells); loss ||x - x*||^2; gradient
    wrt kappa checked on `ncoef` random cells against central differences,
    h = 1e-6, to 1e-6 relative."""
    import torch
    D = DiffusionPattern(*grid)
    kappa = np.exp(gaussian_random_field(D.shape, 1.0, 8.0, seed=20241116))
    rng = np.random.default_rng(7)
    b, xs = rng.standard_normal(D.n), rng.standard_normal(D.n)
    S = P.DeviceSystem(D.matrix(kappa))
    spec = SolveSpec(tol=1e-13, max_iter=5000)
    kap = torch.tensor(kappa, device="cuda", requires_grad=True)
    x = solve(S, D.values(kap), torch.tensor(b, device="cuda"), spec)
    ((x - torch.tensor(xs, device="cuda")) ** 2).sum().backward()
    grad = kap.grad.cpu().numpy()
    cells = rng.choice(D.n, ncoef, replace=False)
    fd = np.array([_fd_gradient(S, D, kappa, b, xs, m, 1e-6, 1e-13) for m in cells])
    err = np.abs(fd - grad[cells]) / np.maximum(np.abs(grad[cells]), 1e-12 * np.abs(grad).max())
    assert err.max() < 1e-6, (err.max(), cells[np.argmax(err)])


def test_adjoint_rejects_nonsymmetric():
    A = P.CSRMatrix.laplacian(8, 8, 1, 0.3, 0.0, 0.0)
    S = P.DeviceSystem(A)
    S.set_precond(P.PRECOND_ILUT, tol=1e-3)
    with pytest.raises(P.PrismError) as e:
        S.adjoint(np.ones(A.n), np.ones(A.n), solver=P.SOLVER_FGMRES, restart=20)
    assert e.value.status == 9


def test_autograd_with_device_refactorisation():
    """SolveSpec(refactor="device"): each forward call recomputes the IC factor on the
    device from the new coefficients (prism_refactor) instead of a new host setup.  The
    loss and gradients equal those of a fresh host factorisation within the solve
    tolerance, and the second call with the same coefficients gives the same loss to the
    last bit (the gradient wrt kappa passes through torch's scatter-add, whose atomic
    order varies between runs: equal to 1e-12)."""
    import torch
    D = DiffusionPattern(10, 9, 8)
    g = gaussian_random_field(D.shape, 1.0, 2.0, seed=5)
    rng = np.random.default_rng(6)
    b0, xs = rng.standard_normal(D.n), rng.standard_normal(D.n)
    S = P.DeviceSystem(D.matrix(np.ones(D.n)))  # factored once on other coefficients
    S.set_precond(P.PRECOND_IC, tol=1e-3)

    def run(spec, system):
        kap = torch.tensor(np.exp(g), dtype=torch.float64, device="cuda", requires_grad=True)
        x = solve(system, D.values(kap), torch.tensor(b0, device="cuda"), spec)
        loss = ((x - torch.tensor(xs, device="cuda")) ** 2).sum()
        loss.backward()
        return loss.item(), kap.grad.cpu().numpy()

    l1, g1 = run(SolveSpec(tol=1e-13, refactor="device"), S)
    l2, g2 = run(SolveSpec(tol=1e-13, refactor="device"), S)
    assert l1 == l2 and rel_err(g1, g2) < 1e-12
    S2 = P.DeviceSystem(D.matrix(np.ones(D.n)))
    l3, g3 = run(SolveSpec(tol=1e-13, refactor=True), S2)
    assert abs(l1 - l3) <= 1e-10 * abs(l3)
    assert rel_err(g1, g3) < 1e-8
