"""CPU checks of the sky oracle: cube-map addressing known answers and the
generator's determinism."""
from __future__ import annotations

import numpy as np

from oracle import sky_oracle


def test_cubemap_face_centres_and_corners(oracle):
    N = 8
    # face centres: +X, -X, +Y, -Y, +Z, -Z
    d = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], float)
    t = oracle.sky_texels(d[:, 0], d[:, 1], d[:, 2], N)
    assert list(t // (N * N)) == [0, 1, 2, 3, 4, 5]
    assert all((t % (N * N)) == (N // 2) * N + N // 2)  # u = v = 1/2 -> texel (N/2, N/2)
    # +Z face: s = x, t = -y: direction (+x, -y) lands in the last column of the last row
    t2 = oracle.sky_texels([0.99], [-0.99], [1.0], N)
    assert t2[0] == (4 * N + (N - 1)) * N + (N - 1)
    # ties go to x, then y
    t3 = oracle.sky_texels([1.0, 0.0], [1.0, 1.0], [0.0, 1.0], N)
    assert t3[0] // (N * N) == 0 and t3[1] // (N * N) == 2


def test_generator_deterministic_and_in_range():
    a = sky_oracle.generate(32, 300, seed=11)
    b = sky_oracle.generate(32, 300, seed=11)
    c = sky_oracle.generate(32, 300, seed=12)
    assert a.shape == (6, 32, 32) and a.dtype == np.float16
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, c)
    noise = a[a < 1]
    assert noise.min() >= 0 and noise.max() < 1 and abs(float(noise.astype(np.float64).mean()) - 0.5) < 0.02
    assert 290 <= int((a >= 2).sum()) <= 300  # stars (a few share a texel)
