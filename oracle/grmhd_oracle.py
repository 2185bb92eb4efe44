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


# ---- packed simulation frames (nubhlight_pack layout) -------------------------

def fnv1a64_hex(blob: bytes) -> str:
    """FNV-1a 64 of the bytes, 16 lower-case hex digits (nubhlight_pack's checksum)."""
    h = 14695981039346656037
    for b in blob:
        h ^= b
        h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return f"{h:016x}"


def write_pack(directory, name: str, samples: np.ndarray, r_range=(2.0, 40.0), channels=("rho", "u", "v1", "v2"),
               checksum: bool = True, bin_key: str = "bin", fmt: str = "RGBA32F", dims=None) -> str:
    """Write a metadata JSON + blob pair in the schema the reference's
    tools/nubhlight_pack.cpp writes; returns the JSON path."""
    import json
    import os

    samples = np.ascontiguousarray(samples, np.float32)
    blob = samples.tobytes()
    with open(os.path.join(directory, name + ".bin"), "wb") as f:
        f.write(blob)
    meta = {"schema_version": 1, "source": "nubhlight", "layout": "channels-last", "format": fmt,
            bin_key: name + ".bin", "grid_dims": list(dims or samples.shape[:3]), "channels": list(channels),
            "min": [float(samples[..., c].min()) for c in range(4)],
            "max": [float(samples[..., c].max()) for c in range(4)], "r_min": r_range[0], "r_max": r_range[1]}
    if checksum:
        meta["checksum_fnv1a64"] = fnv1a64_hex(blob)
    path = os.path.join(directory, name + ".json")
    with open(path, "w") as f:
        json.dump(meta, f, indent=1)
    return path


def _packed_sample(f: np.ndarray, fr, ft, fp):
    nr, nt, np_ = f.shape[:3]
    fr = np.clip(fr, 0, nr - 1)
    ft = np.clip(ft, 0, nt - 1)
    i0 = np.minimum(np.floor(fr).astype(np.int64), max(nr - 2, 0))
    j0 = np.minimum(np.floor(ft).astype(np.int64), max(nt - 2, 0))
    i1, j1 = np.minimum(i0 + 1, nr - 1), np.minimum(j0 + 1, nt - 1)
    tr, tt = fr - i0, ft - j0
    fl = np.floor(fp)
    tp = fp - fl
    k0 = np.mod(fl.astype(np.int64), np_)
    k1 = (k0 + 1) % np_
    acc = np.zeros(fr.shape + (2,))
    for di, ii in ((0, i0), (1, i1)):
        for dj, jj in ((0, j0), (1, j1)):
            for dk, kk in ((0, k0), (1, k1)):
                w = (tr if di else 1 - tr) * (tt if dj else 1 - tt) * (tp if dk else 1 - tp)
                acc += w[..., None] * f[ii, jj, kk, :2].astype(np.float64)
    return acc


def from_packed(left: np.ndarray, right: np.ndarray | None, alpha: float, pr_range, n_r, n_th, n_ph, r_min, r_max,
                n_scale=1e5, theta_scale=10.0, b_scale=30.0) -> np.ndarray:
    """The medium grid sampled from packed frames (grmhd.cu k_grmhd_from_packed)."""
    i = np.arange(n_r)[:, None, None]
    j = np.arange(n_th)[None, :, None]
    k = np.arange(n_ph)[None, None, :]
    r = r_min * np.exp(np.log(r_max / r_min) * i / (n_r - 1)) + 0 * j + 0 * k
    th = (j + 0.5) * (np.pi / n_th) + 0 * i + 0 * k
    ph = k * (2 * np.pi / n_ph) + 0 * i + 0 * j
    pnr, pnt, pnp = left.shape[:3]
    fr = (r - pr_range[0]) / (pr_range[1] - pr_range[0]) * pnr - 0.5
    ft = th / np.pi * pnt - 0.5
    fp = ph / (2 * np.pi) * pnp - 0.5
    a = _packed_sample(left, fr, ft, fp)
    if right is not None:
        b = _packed_sample(right, fr, ft, fp)
        a = a + alpha * (b - a)
    rho, u = a[..., 0], a[..., 1]
    n = np.where(rho > 0, n_scale * rho, 0.0)
    te = np.where(rho > 0, theta_scale * u / np.where(rho > 0, rho, 1.0), 0.0)
    bb = b_scale * np.sqrt(np.maximum(u, 0.0))
    return np.stack([n, te, bb, np.zeros_like(n)], axis=-1).astype(np.float32)
