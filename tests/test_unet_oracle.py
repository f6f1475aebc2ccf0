"""CPU checks of the U-Net oracle itself: the convolution's data and weight
gradients against central finite differences, pooling/upsampling adjoints,
and BF16 rounding (nearest even)."""
from __future__ import annotations

import numpy as np

import unet_oracle as U


def test_conv3_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((3, 4, 5, 2))
    w = rng.standard_normal((27, 3, 2))
    b = rng.standard_normal(3)
    g = rng.standard_normal((3, 4, 5, 3))
    f = lambda x_, w_, b_: float((U.conv3(x_, w_, b_) * g).sum())  # noqa: E731
    dx, dw, db = U.conv3_grad(x, w, g)
    eps = 1e-6
    for _ in range(20):
        idx = tuple(rng.integers(0, s) for s in x.shape)
        xp, xm = x.copy(), x.copy()
        xp[idx] += eps
        xm[idx] -= eps
        assert abs((f(xp, w, b) - f(xm, w, b)) / (2 * eps) - dx[idx]) < 1e-6
        jdx = tuple(rng.integers(0, s) for s in w.shape)
        wp, wm = w.copy(), w.copy()
        wp[jdx] += eps
        wm[jdx] -= eps
        assert abs((f(x, wp, b) - f(x, wm, b)) / (2 * eps) - dw[jdx]) < 1e-6
    assert np.allclose(db, g.sum(axis=(0, 1, 2)))


def test_pool_and_up_are_adjoint_to_their_gradients():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((4, 6, 2, 3))
    y = rng.standard_normal((2, 3, 1, 3))
    assert np.isclose((U.pool(x) * y).sum(), (x * U.pool_grad(y)).sum())
    assert np.isclose((U.up(y) * x).sum(), (y * U.up_grad(x)).sum())


def test_bf16_round_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e38], np.float32)
    r = U.bf16_round(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0 + 2 ** -7) and r[3] == -2.5
