"""Differentiable sparse solve over the C ABI, and the variable-coefficient
diffusion model problem it is checked on.

``solve(system, values, b)`` returns x = A(values)^{-1} b as a torch tensor.
Its backward pass is the library's adjoint solve (prism_adjoint_solve_device):
one solve with A^T (= A for the symmetric operators supported) and the same
preconditioner gives dL/db = lambda = A^{-T} dL/dx, and the outer product
dL/dA_ij = -lambda_i x_j sampled on A's stored pattern gives dL/dvalues.
Everything upstream of ``values`` (for instance the assembly of A from cell
coefficients below) is differentiated by torch as usual.

The diffusion operator: a cell-centred 7-point finite-volume discretisation
of -div(kappa grad u) on an nx x ny x nz grid of unit cells, face
coefficients the harmonic mean of the two cells, homogeneous Dirichlet
boundaries through a ghost cell carrying the boundary cell's kappa.  Its
pattern is the one of generateLaplacianCSR(nx, ny, nz)
(source/MatrixClass/ModelProblem.cpp:68-133), so the values line up with
that CSR entry for entry.
"""
from __future__ import annotations

import numpy as np

from . import (CSRMatrix, DeviceSystem, PRECOND_IC, PRISM_FP64, SOLVER_FCG)


class SolveSpec:
    """How the forward and adjoint solves run: solver, tolerance, and whether the
    preconditioner is refactored from the new values on every forward call
    (refactor=True: a new host setup; "device": the IC / ILDLT factor recomputed on
    the device on its own pattern, prism_refactor; False: the caller's preconditioner
    stays)."""

    def __init__(self, solver=SOLVER_FCG, tol=1e-12, max_iter=5000, restart=0, precond=PRECOND_IC,
                 precond_tol=1e-3, precision=PRISM_FP64, refactor=True):
        self.solver, self.tol, self.max_iter, self.restart = solver, tol, max_iter, restart
        self.precond, self.precond_tol, self.precision, self.refactor = precond, precond_tol, precision, refactor


def _function():
    import torch

    class SparseSolve(torch.autograd.Function):
        @staticmethod
        def forward(ctx, values, b, system, spec):
            v = values.detach().contiguous()
            system.update_values(v)
            if spec.refactor == "device":
                system.refactor()
            elif spec.refactor:  # otherwise the caller's preconditioner stays (a stale one still gives the exact x)
                system.set_precond(spec.precond, tol=spec.precond_tol, precision=spec.precision)
            x, st = system.solve(b.detach().contiguous(), solver=spec.solver, tol=spec.tol, max_iter=spec.max_iter,
                                 restart=spec.restart)
            if not st.converged:
                raise RuntimeError(f"forward solve did not converge ({st.num_iter} iterations, "
                                   f"error {st.final_error:.3e})")
            ctx.system, ctx.spec = system, spec
            ctx.save_for_backward(v, x)
            return x

        @staticmethod
        def backward(ctx, gx):
            v, x = ctx.saved_tensors
            system, spec = ctx.system, ctx.spec
            system.update_values(v)  # the operator of this forward call, whatever ran since
            lam, gv, st = system.adjoint(gx.contiguous(), x, solver=spec.solver, tol=spec.tol,
                                         max_iter=spec.max_iter, restart=spec.restart)
            if not st.converged:
                raise RuntimeError(f"adjoint solve did not converge ({st.num_iter} iterations)")
            return (gv if ctx.needs_input_grad[0] else None, lam if ctx.needs_input_grad[1] else None, None, None)

    return SparseSolve


_FN = None


def solve(system: DeviceSystem, values, b, spec: SolveSpec | None = None):
    """x = A^{-1} b with A = (system's pattern, values); differentiable in values and b."""
    global _FN
    if _FN is None:
        _FN = _function()
    return _FN.apply(values, b, system, spec or SolveSpec())


# =============================================================================
# Variable-coefficient diffusion model problem
# =============================================================================
class DiffusionPattern:
    """Index maps from cell coefficients to the CSR values of the 7-point pattern."""

    def __init__(self, nx: int, ny: int, nz: int):
        self.shape = (nx, ny, nz)
        self.A0 = CSRMatrix.laplacian(nx, ny, nz)
        n = nx * ny * nz
        rp, ci = self.A0.rowptr.astype(np.int64), self.A0.col.astype(np.int64)
        rows = np.repeat(np.arange(n), np.diff(rp))
        # cell index = i + nx * (j + ny * k)
        idx = np.arange(n).reshape(nz, ny, nx)
        fa, fb = [], []
        for axis in range(3):
            a = np.take(idx, np.arange(idx.shape[axis] - 1), axis=axis).ravel()
            bb = np.take(idx, np.arange(1, idx.shape[axis]), axis=axis).ravel()
            fa.append(a)
            fb.append(bb)
        self.face_a = np.concatenate(fa)
        self.face_b = np.concatenate(fb)
        # boundary faces: every cell face that leaves the grid, one entry per (cell, face)
        bnd = []
        for axis in range(3):
            first = np.take(idx, [0], axis=axis).ravel()
            last = np.take(idx, [idx.shape[axis] - 1], axis=axis).ravel()
            bnd += [first, last]
        self.bnd_cell = np.concatenate(bnd)
        # CSR positions of (a, b), (b, a) and the diagonal
        key = rows * n + ci
        order = np.argsort(key)
        skey = key[order]

        def pos(r, c):
            k = r * n + c
            p = np.searchsorted(skey, k)
            if not np.array_equal(skey[p], k):
                raise ValueError("entry outside the 7-point pattern")
            return order[p]

        self.pos_ab = pos(self.face_a, self.face_b)
        self.pos_ba = pos(self.face_b, self.face_a)
        self.pos_diag = pos(np.arange(n), np.arange(n))
        self.n, self.nnz = n, self.A0.nnz

    def values(self, kappa):
        """CSR values of A(kappa) for kappa a torch tensor of nx*ny*nz cell
        coefficients (cell index i + nx*(j + ny*k)); differentiable."""
        import torch
        dev = kappa.device
        ta = torch.as_tensor(self.face_a, device=dev)
        tb = torch.as_tensor(self.face_b, device=dev)
        ka, kb = kappa[ta], kappa[tb]
        kf = 2.0 * ka * kb / (ka + kb)
        diag = torch.zeros(self.n, dtype=kappa.dtype, device=dev)
        diag = diag.index_add(0, ta, kf).index_add(0, tb, kf)
        tbc = torch.as_tensor(self.bnd_cell, device=dev)
        diag = diag.index_add(0, tbc, kappa[tbc])
        v = torch.zeros(self.nnz, dtype=kappa.dtype, device=dev)
        v = v.index_put((torch.as_tensor(self.pos_ab, device=dev),), -kf)
        v = v.index_put((torch.as_tensor(self.pos_ba, device=dev),), -kf)
        v = v.index_put((torch.as_tensor(self.pos_diag, device=dev),), diag)
        return v

    def matrix(self, kappa_np: np.ndarray) -> CSRMatrix:
        import torch
        v = self.values(torch.from_numpy(np.asarray(kappa_np, np.float64))).numpy()
        return CSRMatrix(self.A0.rowptr, self.A0.col, v)


def gaussian_random_field(shape, sigma: float = 1.0, corr_len: float = 8.0, seed: int = 0) -> np.ndarray:
    """Stationary Gaussian field on a periodic grid of `shape` (nz, ny, nx order of
    the returned array is x fastest, flattened as i + nx*(j + ny*k)), squared-
    exponential covariance exp(-r^2 / (2 corr_len^2)), standard deviation sigma:
    white noise filtered in Fourier space, rescaled to the requested sigma."""
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((nz, ny, nx))
    kz = np.fft.fftfreq(nz)[:, None, None]
    ky = np.fft.fftfreq(ny)[None, :, None]
    kx = np.fft.fftfreq(nx)[None, None, :]
    k2 = (2 * np.pi) ** 2 * (kx ** 2 + ky ** 2 + kz ** 2)
    filt = np.exp(-k2 * corr_len ** 2 / 4.0)  # square root of the covariance spectrum
    g = np.real(np.fft.ifftn(np.fft.fftn(w) * filt))
    g -= g.mean()
    g *= sigma / g.std()
    return g.ravel()
