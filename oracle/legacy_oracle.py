"""Numpy restatement of the legacy RGBA layer (test infrastructure only).

Mirrors blackhole_b200/csrc/host/legacy_api.cpp, device/legacy.cu and
device/postprocess.cu: the camera derived from BH_LaunchParams, the blackbody
colour table, the disk / background shading, the bridge's post-processing
(bloom, exposure, vignette, ACES, gamma: src/blender_bridge/cuda_postprocess.cu),
the lensing-map channels and the disk emission texture. Geometry (which pixel hits what) comes from the C++ oracle
(pyoracle.Oracle.trace_camera / trace_pixels); only tests import this.
"""
from __future__ import annotations

import math

import numpy as np

from blackhole_b200._abi import default_scene

BB_N = 256
BB_LOG2_T0 = np.float32(8.643856189774724)   # log2(400)
BB_LOG2_T1 = np.float32(15.609640474436812)  # log2(50000)
DISK_PEAK_T = 10000.0


def _lobe(x, mu, s1, s2):
    t = (x - mu) / np.where(x < mu, s1, s2)
    return np.exp(-0.5 * t * t)


def blackbody_table() -> np.ndarray:
    """[256][3] linear-sRGB chromaticity (Y = 1): Planck x CIE 1931 (multi-lobe
    Gaussian fit of Wyman, Sloan & Shirley 2013), 360-830 nm, sRGB matrix."""
    lam = np.arange(360, 831, dtype=np.float64)
    xb = 1.056 * _lobe(lam, 599.8, 37.9, 31.0) + 0.362 * _lobe(lam, 442.0, 16.0, 26.7) - \
        0.065 * _lobe(lam, 501.1, 20.4, 26.2)
    yb = 0.821 * _lobe(lam, 568.8, 46.9, 40.5) + 0.286 * _lobe(lam, 530.9, 16.3, 31.1)
    zb = 1.217 * _lobe(lam, 437.0, 11.8, 36.0) + 0.681 * _lobe(lam, 459.0, 26.0, 13.8)
    out = np.zeros((BB_N, 3))
    for i in range(BB_N):
        T = 2.0 ** (float(BB_LOG2_T0) + (float(BB_LOG2_T1) - float(BB_LOG2_T0)) * i / (BB_N - 1))
        B = 1.0 / (lam ** 5 * np.expm1(1.438776877e7 / (lam * T)))
        X, Y, Z = (B * xb).sum(), (B * yb).sum(), (B * zb).sum()
        X, Z, Y = X / Y, Z / Y, 1.0
        rgb = np.array([3.2406 * X - 1.5372 * Y - 0.4986 * Z, -0.9689 * X + 1.8758 * Y + 0.0415 * Z,
                        0.0557 * X - 0.2040 * Y + 1.0570 * Z])
        out[i] = np.maximum(rgb, 0.0)
    return out.astype(np.float32)


def blackbody(t: np.ndarray, tab: np.ndarray) -> np.ndarray:
    t = np.asarray(t, np.float32)
    x = (np.log2(np.maximum(t, np.float32(1))) - BB_LOG2_T0) / (BB_LOG2_T1 - BB_LOG2_T0) * np.float32(BB_N - 1)
    x = np.clip(x, 0, BB_N - 1)
    i = np.minimum(x.astype(np.int64), BB_N - 2)
    w = (x - i)[..., None]
    return tab[i] * (1 - w) + tab[i + 1] * w


def aces(x):
    y = (x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14)
    return np.clip(y, 0.0, 1.0)


def camera(p) -> tuple[dict, np.ndarray, np.ndarray]:
    """(scene keyword arguments, cam_f64[17], cam_i32[2]) of a LaunchParams,
    as legacy_api.cpp camera_job derives them."""
    m = 0.5 * float(p.rs)
    x, y, z = (float(v) / m for v in p.cam_pos)
    r0 = math.sqrt(x * x + y * y + z * z)
    u0 = z / r0
    spin = float(p.spin) if p.kerr_enabled else 0.0
    max_dist = float(p.max_dist) / m
    scene = dict(spin=spin, r_obs=r0, theta_obs=min(max(math.acos(max(-1.0, min(1.0, u0))), 1e-9), math.pi - 1e-9),
                 width=p.width, height=p.height, integrator=1, precision=0, potential_form=1, max_crossings=1,
                 max_steps=p.max_steps, escape_factor=max(max_dist, 1.01 * r0) / r0,
                 disk_r_in=float(p.isco) / m if p.isco > 0 else 0.0,
                 disk_r_out=30.0 * float(p.rs) / m if p.adisk_enabled else 1e-9)
    B = np.array(p.cam_basis, np.float64)
    rho = math.hypot(x, y)
    cf = np.concatenate([B[0:3], B[3:6], B[6:9],
                         [float(p.fov_scale), p.width / p.height, float(p.frame_shift_x), float(p.frame_shift_y),
                          r0, u0, x / rho if rho > 0 else 1.0, y / rho if rho > 0 else 0.0]])
    return scene, cf, np.array([p.width, p.height], np.int32)


def scene_of(kw: dict):
    s = default_scene(width=kw["width"], height=kw["height"], spin=kw["spin"], theta_obs=kw["theta_obs"],
                      integrator=kw["integrator"], max_crossings=kw["max_crossings"], precision=kw["precision"])
    s.r_obs = kw["r_obs"]
    s.potential_form = kw["potential_form"]
    s.max_steps = kw["max_steps"]
    s.escape_factor = kw["escape_factor"]
    s.disk_r_in = kw["disk_r_in"]
    s.disk_r_out = kw["disk_r_out"]
    return s


def shade(fields: dict, p, cphi: float, sphi: float, tab=None) -> np.ndarray:
    """RGBA [n][4] of legacy.cu k_legacy_shade without textures (black background)."""
    tab = blackbody_table() if tab is None else tab
    cls = fields["cls"]
    n = cls.size
    g = fields["g"][0] if fields["g"].ndim == 2 else fields["g"]
    F = fields["flux"].astype(np.float32)
    gg = (g.astype(np.float32) if p.redshift_enabled else np.ones(n, np.float32))
    t = np.float32(DISK_PEAK_T) * gg * np.sqrt(np.sqrt(F))
    inten = np.float32(p.adisk_lit) * (gg * gg) * (gg * gg) * F
    col = blackbody(t, tab) * inten[:, None]
    col[cls != 1] = 0.0
    return np.concatenate([col, np.ones((n, 1), np.float32)], axis=1)


def _blur(img: np.ndarray, r: int, axis: int) -> np.ndarray:
    """Normalized Gaussian of half-width r, sigma = r / 2, clamped edges
    (cuda_postprocess.cu:42-98), along one axis of an [h, w, 3] image."""
    dx = np.arange(-r, r + 1)
    g = np.exp(-(dx * dx) / (2.0 * (0.5 * r) ** 2))
    g /= g.sum()
    n = img.shape[axis]
    out = np.zeros_like(img)
    for k, d in enumerate(dx):
        idx = np.clip(np.arange(n) + d, 0, n - 1)
        out += g[k] * np.take(img, idx, axis=axis)
    return out


def postprocess(fb: np.ndarray, threshold: float, strength: float, exposure: float) -> np.ndarray:
    """bhb_cuda_postprocess of an [h, w, 4] framebuffer (cuda_postprocess.cu:237-275):
    bright-pass, blur at half-widths 4, 8, 16, 32 of that same bright-pass,
    summed and added times the strength; then exposure, vignette, ACES,
    gamma 1/2.2, with red and blue read at (int(u w), int(v h)) of the
    float32 uv. Float64 arithmetic except the uv and that index."""
    h, w = fb.shape[:2]
    col = fb[..., :3].astype(np.float64)
    if strength != 0.0:
        lum = 0.2126 * col[..., 0] + 0.7152 * col[..., 1] + 0.0722 * col[..., 2]
        scale = np.where(lum > 0.001, np.maximum(0.0, lum - threshold) / np.where(lum > 0.001, lum, 1.0), 0.0)
        bright = col * scale[..., None]
        acc = np.zeros_like(col)
        for r in (4, 8, 16, 32):
            acc += _blur(_blur(bright, r, 1), r, 0)
        col = col + strength * acc
    f32 = np.float32
    u = np.arange(w, dtype=f32) / f32(w)
    v = np.arange(h, dtype=f32) / f32(h)
    rx = np.clip(np.floor(u * f32(w)).astype(np.int64), 0, w - 1)
    ry = np.clip(np.floor(v * f32(h)).astype(np.int64), 0, h - 1)
    red = col[ry[:, None], rx[None, :], 0]
    blue = col[ry[:, None], rx[None, :], 2]
    out = np.stack([red, col[..., 1], blue], axis=-1)
    uu, vv = np.meshgrid(u.astype(np.float64), v.astype(np.float64))
    d2 = (uu - 0.5) ** 2 + (vv - 0.5) ** 2
    vig = np.sqrt(np.maximum(1.0 - d2 * 0.5, 0.0))
    out = aces(out * exposure * vig[..., None])
    out = np.maximum(out, 0.0) ** (1.0 / 2.2)
    return np.concatenate([out, np.ones((h, w, 1))], axis=-1)


def lensing(fields: dict) -> np.ndarray:
    cls = fields["cls"]
    r = fields["r_hit"][0]
    g = fields["g"][0]
    out = np.zeros((cls.size, 4))
    hit = cls == 1
    out[:, 1] = 1.0
    out[:, 3] = 1.0
    out[hit, 0] = np.sqrt(np.maximum(0.0, 1.0 - 2.0 / r[hit]))
    out[hit, 1] = g[hit]
    out[hit, 2] = 1.0
    out[(cls != 1) & (cls != 0), 0] = 1.0
    return out


def disk_texture(a: float, r_isco: float, r_out: float, flux_peak: float, incl: float, w: int, h: int,
                 tab=None) -> np.ndarray:
    tab = blackbody_table() if tab is None else tab
    iy, ix = np.meshgrid(np.arange(h), np.arange(w), indexing="ij")
    r = r_isco + (r_out - r_isco) * iy / h
    phi = 2 * np.pi * ix / w
    t = 1.0 - np.sqrt(r_isco / r)
    F = np.minimum(1.0, np.maximum(t, 0.0) / r ** 3 / flux_peak)
    F[r < r_isco] = 0.0
    lam = -r * np.sin(phi) * math.sin(incl)
    x = np.sqrt(r)
    v = x ** 3 * (x ** 3 - 3 * x + 2 * a)
    g = np.where(v > 0, np.sqrt(np.maximum(v, 0)) / (x ** 3 + a - lam), 0.0)
    tn = np.sqrt(np.sqrt(F)).astype(np.float32)
    col = blackbody(np.float32(DISK_PEAK_T) * g.astype(np.float32) * tn, tab)
    inten = (g ** 4 * F).astype(np.float32)
    return np.concatenate([col * inten[..., None], tn[..., None]], axis=-1)
