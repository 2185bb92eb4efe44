"""CPU checks of the surrogate network's oracle and host-side layout.

The oracle (oracle/surrogate_oracle.py) is what the GPU forward and backward
kernels are compared with; here it is itself checked against central finite
differences of its loss, and its BF16 rounding against known values.
"""
from __future__ import annotations

import numpy as np

from oracle import surrogate_oracle as so


def random_params(rng, scale=0.3):
    n = sum(k * nn + nn for k, nn in zip(so.LAYER_K, so.LAYER_N))
    return rng.normal(0.0, scale, n) / 8.0


def random_targets(rng, B):
    t = np.zeros((B, 16))
    t[:, 0] = rng.integers(-1, 3, B)
    t[:, 1] = rng.integers(0, 3, B)
    t[:, 1] = np.where(t[:, 0] == 1, np.maximum(t[:, 1], 1), np.where(t[:, 0] >= 0, 0, t[:, 1] * 0))
    t[:, 2:12] = rng.normal(0.0, 0.5, (B, 10))
    return t


def test_bf16_rounding_known_values():
    vals = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 3.0e-30, 65504.0], np.float64)
    got = so.bf16(vals)
    assert got[0] == 1.0
    assert got[1] == 1.0                      # tie -> even
    assert got[2] == 1.0 + 2.0 ** -6          # 1 + 3/256 -> 1 + 4/256 (tie -> even mantissa)
    assert got[3] == -2.5
    assert abs(got[4] - 3.0e-30) / 3.0e-30 < 2.0 ** -8
    assert got[5] == 65536.0


def test_param_layout_matches_library(lib):
    assert lib.bh_surrogate_param_count() == sum(k * n + n for k, n in zip(so.LAYER_K, so.LAYER_N)) == 250896


def test_features_shape_and_padding():
    rng = np.random.default_rng(0)
    x = np.stack([rng.uniform(-15, 15, 50), rng.uniform(-15, 15, 50), rng.uniform(0, 0.998, 50),
                  np.cos(np.radians(rng.uniform(5, 89, 50)))], 1)
    F = so.features(x)
    assert F.shape == (50, 192)
    assert np.all(F[:, 134:] == 0.0)
    np.testing.assert_allclose(F[:, 0] ** 2 + F[:, 1] ** 2, 1.0, rtol=1e-12)
    np.testing.assert_allclose(F[:, 128], x[:, 0] / 15.0)


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    B = 24
    params = random_params(rng)
    x = np.stack([rng.uniform(-15, 15, B), rng.uniform(-15, 15, B), rng.uniform(0, 0.998, B),
                  np.cos(np.radians(rng.uniform(5, 89, B)))], 1)
    F = so.features(x)
    tg = random_targets(rng, B)
    out, cache = so.forward(params, F, emulate=False)
    _, dout = so.loss_and_grad(out, tg)
    g = so.backward(params, cache, dout, emulate=False)
    offs = np.cumsum([0] + [k * n + n for k, n in zip(so.LAYER_K, so.LAYER_N)])
    idx = []
    for l in range(5):
        k, n = so.LAYER_K[l], so.LAYER_N[l]
        w = rng.integers(0, n, 4) * k + rng.integers(0, 134 if l == 0 else k, 4)
        idx += list(offs[l] + w) + list(offs[l] + n * k + rng.integers(0, n, 2))
    h = 1e-6
    for i in idx:
        p1, p0 = params.copy(), params.copy()
        p1[i] += h
        p0[i] -= h
        fd = (so.total_loss(p1, F, tg) - so.total_loss(p0, F, tg)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-7, (i, fd, g[i])
