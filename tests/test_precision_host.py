"""Precision argument of the host-side factor builders (no device needed):
PRISM_FP32_APPLY builds the same float factor as PRISM_FP32 (only the
device sweeps' arithmetic differs), and values outside the enum are
rejected with an error naming the precision."""
from __future__ import annotations

import numpy as np
import pytest

import prispack_b200 as P


@pytest.mark.parametrize("kind", [P.PRECOND_IC, P.PRECOND_ILDLT, P.PRECOND_ILUT])
def test_fp32_apply_factor_equals_fp32_factor(kind):
    A = P.CSRMatrix.laplacian(9, 8, 7) if kind != P.PRECOND_ILUT else P.CSRMatrix.convection_diffusion(9, 8, 7, 4.0, 2.0, 1.0)
    f32 = P.HostFactor(A, kind, tol=1e-3, precision=P.PRISM_FP32)
    fa = P.HostFactor(A, kind, tol=1e-3, precision=P.PRISM_FP32_APPLY)
    assert f32.info() == fa.info()
    for which in (0, 1) if kind == P.PRECOND_ILUT else (0,):
        for a, b in zip(f32.arrays(which), fa.arrays(which)):
            np.testing.assert_array_equal(a, b)


def test_fp32_apply_amsed_setup_equals_fp32():
    A = P.CSRMatrix.laplacian(12, 12, 12)
    kw = dict(levels=3, lanczos_steps=16, low_rank=8, lowrank_type=0, reorder=0)
    h32 = P.HostAmsed(A, precision=P.PRISM_FP32, **kw)
    ha = P.HostAmsed(A, precision=P.PRISM_FP32_APPLY, **kw)
    i32, ia = h32.info(), ha.info()
    assert i32["mnnz"] == ia["mnnz"] and i32["nlev"] == ia["nlev"]
    np.testing.assert_array_equal(i32["lev_ptr"], ia["lev_ptr"])
    np.testing.assert_array_equal(h32.perm(), ha.perm())


@pytest.mark.parametrize("bad", [-1, 3, 7])
def test_precision_out_of_range(bad):
    A = P.CSRMatrix.laplacian(5, 5, 1)
    with pytest.raises(P.PrismError, match="precision"):
        P.HostFactor(A, P.PRECOND_IC, precision=bad)
    with pytest.raises(P.PrismError, match="precision"):
        P.HostAmsed(A, precision=bad, levels=2, lanczos_steps=4, low_rank=2, lowrank_type=0, reorder=0)
