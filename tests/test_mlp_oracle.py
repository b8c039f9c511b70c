"""Pin of the FP64 MLP oracle: its analytic gradient against central finite
differences (no bf16 rounding), and its bf16 rounding against the format."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import mlp_oracle as mo  # noqa: E402


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    dims = (8, 16, 8, 3)
    n = sum(dims[i] * dims[i + 1] + dims[i + 1] for i in range(len(dims) - 1))
    p = rng.standard_normal(n) * 0.3
    x = rng.standard_normal((5, dims[0]))
    t = rng.standard_normal((5, dims[-1]))
    _, g = mo.loss_and_grad(p, dims, x, t, round_bf16=False)
    for k in rng.choice(n, 25, replace=False):
        e = np.zeros(n)
        e[k] = 1e-6
        lp, _ = mo.loss_and_grad(p + e, dims, x, t, round_bf16=False)
        lm, _ = mo.loss_and_grad(p - e, dims, x, t, round_bf16=False)
        assert abs((lp - lm) / 2e-6 - g[k]) <= 1e-6 * max(1.0, abs(g[k]))


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.001953125, 3.14159265, -2.5e-3, 1.01171875], dtype=np.float32)
    r = mo.bf16(v)
    # 1 + 2^-8 and 1 + 3*2^-8 are halfway cases: ties go to the even mantissa
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 and r[5] == 1.015625
    assert abs(r[3] - 3.140625) < 1e-12
    assert abs(r[4] + 0.0025024414) < 1e-9
