"""Closed-form Kerr null-geodesic helpers (include/bh_analytic.h) from Python.

Thin ctypes wrappers over the library's host entry points, the counterparts of
the reference's src/physics/analytic_kerr_geodesic.h and
src/cuda/device_analytic_kerr.cuh helpers. M = 1; lambda is Mino time.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._abi import load_library

MOTION = {0: "transit", 1: "plunge", 2: "scatter", 3: "orbit", 4: "invalid"}


def _lib() -> C.CDLL:
    lib = load_library()
    if getattr(lib, "_analytic_declared", False):
        return lib
    d, vp = C.c_double, C.c_void_p
    for name, args, res in (
            ("bh_analytic_radial_potential", [d, d, d, d], d),
            ("bh_analytic_quartic_coeffs", [d, d, d, vp], None),
            ("bh_analytic_radial_roots", [d, d, d, vp, vp, C.POINTER(C.c_int)], C.c_int),
            ("bh_analytic_r_bound", [d, vp, d], d),
            ("bh_analytic_radial_half_period", [vp], d),
            ("bh_analytic_critical_impact_params", [d, d, vp], None),
            ("bh_analytic_prograde_photon_orbit", [d], d),
            ("bh_analytic_retrograde_photon_orbit", [d], d),
            ("bh_analytic_ellpj", [d, d, vp], None),
            ("bh_analytic_ellint_k", [d], d)):
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    lib._analytic_declared = True
    return lib


def radial_potential(r: float, a: float, xi: float, eta: float) -> float:
    return _lib().bh_analytic_radial_potential(r, a, xi, eta)


def quartic_coeffs(a: float, xi: float, eta: float) -> tuple[float, float, float]:
    out = np.zeros(3)
    _lib().bh_analytic_quartic_coeffs(a, xi, eta, out.ctypes.data)
    return tuple(out)


def radial_roots(c2: float, c1: float, c0: float) -> tuple[np.ndarray, int, str]:
    """(roots as complex [4], real ones first and descending; n_real; motion label)."""
    re, im = np.zeros(4), np.zeros(4)
    motion = C.c_int()
    n = _lib().bh_analytic_radial_roots(c2, c1, c0, re.ctypes.data, im.ctypes.data, C.byref(motion))
    return re + 1j * im, n, MOTION.get(motion.value, "invalid")


def r_bound(lam: float, roots_desc, lam0: float = 0.0) -> float:
    r = np.ascontiguousarray(roots_desc, np.float64)
    return _lib().bh_analytic_r_bound(lam, r.ctypes.data, lam0)


def radial_half_period(roots_desc) -> float:
    r = np.ascontiguousarray(roots_desc, np.float64)
    return _lib().bh_analytic_radial_half_period(r.ctypes.data)


def critical_impact_params(r_ph: float, a: float) -> tuple[float, float]:
    out = np.zeros(2)
    _lib().bh_analytic_critical_impact_params(r_ph, a, out.ctypes.data)
    return out[0], out[1]


def prograde_photon_orbit(a: float) -> float:
    return _lib().bh_analytic_prograde_photon_orbit(a)


def retrograde_photon_orbit(a: float) -> float:
    return _lib().bh_analytic_retrograde_photon_orbit(a)


def ellpj(u: float, m: float) -> tuple[float, float, float]:
    out = np.zeros(3)
    _lib().bh_analytic_ellpj(u, m, out.ctypes.data)
    return tuple(out)


def ellint_k(k: float) -> float:
    return _lib().bh_analytic_ellint_k(k)
