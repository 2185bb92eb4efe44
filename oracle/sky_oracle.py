"""CPU oracle of the background sky cubemap (test infrastructure only).

Restates the seeded sky of bh_sky_generate (blackhole_b200/csrc/device/sky.cuh,
csrc/host/sky.cpp): texel k holds the top 24 bits of
splitmix64(seed * 0x100000001B3 + k) (Steele, Lea & Flood 2014) scaled by
2^-24 and rounded to FP16; star s (s = 0 .. n_stars-1) lands on texel
splitmix64((seed ^ 0x5354415253) + 2s) mod 6N^2 with brightness
2 + 18 u, u the top 24 bits of splitmix64((seed ^ 0x5354415253) + 2s + 1)
scaled by 2^-24, added in FP32 to the texel's noise (stars of one texel in
star order) before the FP16 rounding. The reference has no generated sky:
its backgrounds are image textures bound to GL (unavailable here).
"""
from __future__ import annotations

import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = (np.asarray(x, np.uint64) + np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def noise(seed: int, k: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        x = np.uint64(seed) * np.uint64(0x100000001B3) + np.asarray(k, np.uint64)
    return (splitmix64(x) >> np.uint64(40)).astype(np.float32) * np.float32(1.0 / 16777216.0)


def generate(size: int, n_stars: int, seed: int) -> np.ndarray:
    """FP16 cubemap [6][size][size]."""
    n = 6 * size * size
    tex = noise(seed, np.arange(n, dtype=np.uint64))
    base = np.uint64(seed) ^ np.uint64(0x5354415253)
    stars: dict[int, np.float32] = {}
    for s in range(n_stars):
        with np.errstate(over="ignore"):
            h1 = int(splitmix64(base + np.uint64(2 * s)))
            h2 = int(splitmix64(base + np.uint64(2 * s + 1)))
        k = h1 % n
        b = np.float32(2.0) + np.float32(18.0) * (np.float32(h2 >> 40) * np.float32(1.0 / 16777216.0))
        if k in stars:
            stars[k] = np.float32(stars[k] + b)
        else:
            stars[k] = np.float32(tex[k] + b)
    for k, v in stars.items():
        tex[k] = v
    return tex.astype(np.float16).reshape(6, size, size)
