"""CPU oracle of the synthetic volumetric medium (test infrastructure only).

Restates bh_grmhd_synthetic (include/bh_rt.h): a Gaussian torus times exp of
a Gaussian random field written as M = 256 random Fourier modes
(sigma sqrt(2/M) sum cos(k.x + phase), k ~ N(0, I / l^2): Rahimi & Recht
2007 random features of the Gaussian kernel), drawn from a splitmix64
stream (Steele, Lea & Flood 2014) through the Box-Muller transform.
"""
from __future__ import annotations

import numpy as np

from .sky_oracle import splitmix64

MODES = 256


def modes(seed: int, corr_len: float) -> np.ndarray:
    base = np.uint64(seed) ^ np.uint64(0x4752464D4F444553)
    count = [0]

    def nxt() -> float:
        with np.errstate(over="ignore"):
            h = int(splitmix64(base + np.uint64(count[0])))
        count[0] += 1
        return float(h >> 11) * (1.0 / 9007199254740992.0)

    out = np.zeros((MODES, 4))
    for m in range(MODES):
        z = []
        for _ in range(2):
            u1 = 1.0 - nxt()
            u2 = nxt()
            rad = np.sqrt(-2.0 * np.log(u1))
            z += [rad * np.cos(2 * np.pi * u2), rad * np.sin(2 * np.pi * u2)]
        out[m, :3] = np.array(z[:3]) / corr_len
        out[m, 3] = 2 * np.pi * nxt()
    return out


def grid(n_r, n_th, n_ph, r_min, r_max, r_in=6.0, r_peak=12.0, width=3.0, n0=1e5, theta0=20.0, b0=30.0,
         sigma=0.5, corr_len=2.0, seed=1) -> np.ndarray:
    """float32 [n_r][n_th][n_ph][4] = (n_e, Theta_e, |B|, 0)."""
    md = modes(seed, corr_len)
    i = np.arange(n_r)[:, None, None]
    j = np.arange(n_th)[None, :, None]
    k = np.arange(n_ph)[None, None, :]
    r = r_min * np.exp(np.log(r_max / r_min) * i / (n_r - 1))
    th = (j + 0.5) * np.pi / n_th
    ph = k * 2 * np.pi / n_ph
    st, ct = np.sin(th), np.cos(th)
    x, y, z = r * st * np.cos(ph), r * st * np.sin(ph), r * ct * np.ones_like(ph)
    f = np.zeros(np.broadcast(x, y, z).shape)
    for m in range(MODES):
        f += np.cos(md[m, 0] * x + md[m, 1] * y + md[m, 2] * z + md[m, 3])
    f *= sigma * np.sqrt(2.0 / MODES)
    R = r * st
    t = np.exp(-((R - r_peak) ** 2 + z ** 2) / (2 * width ** 2))
    t = np.where(r < r_in, t * np.exp(-(r_in - r) ** 2), t)
    n = n0 * t * np.exp(f)
    out = np.zeros(n.shape + (4,), np.float32)
    out[..., 0] = n
    out[..., 1] = np.broadcast_to(theta0 * r_peak / r, n.shape)
    out[..., 2] = b0 * np.sqrt(n / n0)
    return out
