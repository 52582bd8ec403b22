"""The oracle's single-precision sweep (orc_sweep_f32, the arithmetic of the
single-precision apply, PRISM_FP32_APPLY): bit-exact against a plain
float32 loop, and within single-precision accuracy of the double sweep."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as orc
from test_stream_layout import random_triangular, substitute


def f32_loop(rp, ci, v, diag, op, lower, b):
    n = len(rp) - 1
    x = [np.float32(0)] * n
    rows = range(n) if lower else range(n - 1, -1, -1)
    for r in rows:
        s = np.float32(0)
        for k in range(rp[r], rp[r + 1]):
            s = np.float32(s + np.float32(np.float32(v[k]) * x[ci[k]]))
        bb = np.float32(b[r])
        d = np.float32(diag[r]) if diag is not None else np.float32(1)
        if op == 0:
            res = np.float32(np.float32(bb - s) / d)
        elif op == 1:
            res = np.float32(np.float32(bb - s) * d)
        elif op == 2:
            res = np.float32(bb - s)
        else:
            res = np.float32(np.float32(bb / d) - s)
        x[r] = res
    return np.array(x, np.float64)


@pytest.mark.parametrize("lower", [True, False])
@pytest.mark.parametrize("op", [0, 1, 2, 3])
def test_sweep_f32_bit_exact_and_close_to_double(lower, op):
    rng = np.random.default_rng(300 + op + 10 * lower)
    n = 257
    rp, ci, v = random_triangular(n, lower, rng)
    diag = rng.uniform(1.0, 2.0, n)
    b = rng.standard_normal(n)
    d = diag if op != 2 else None
    got = orc.sweep_f32(rp, ci, v, b, diag=d, op=op, lower=lower)
    np.testing.assert_array_equal(got, f32_loop(rp, ci, v, d, op, lower, b))
    want = substitute(rp, ci, v, diag, op, lower, b)
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-5
