"""include/bh_analytic.h on the CPU: the reference's golden cases for its
analytic helpers (tests/analytic_geodesic_reproducibility_test.cpp:1-200,
tests/cuda_analytic_kerr_test.cu:136-267), agreement with the reference's own
src/physics/analytic_kerr_geodesic.h compiled unmodified
(oracle/_ref/libbh_ref_analytic.so) where that is correct, and the Jacobi and
elliptic functions against scipy / 30-digit mpmath."""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import mpmath as mp
import numpy as np
import pytest
import scipy.special as sp
from scipy import integrate

REF = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libbh_ref_analytic.so"


@pytest.fixture(scope="module")
def an(lib):
    from blackhole_b200 import analytic

    return analytic


@pytest.fixture(scope="module")
def ref():
    if not REF.exists():
        pytest.skip("reference analytic build absent (oracle/_ref)")
    L = C.CDLL(str(REF))
    d, vp = C.c_double, C.c_void_p
    L.ref_radial_potential.argtypes = [d, d, d, d]
    L.ref_radial_potential.restype = d
    L.ref_quartic_coeffs.argtypes = [d, d, d, vp]
    L.ref_radial_roots.argtypes = [d, d, d, vp, vp, C.POINTER(C.c_int)]
    L.ref_critical_impact_params.argtypes = [d, d, vp]
    for f in (L.ref_prograde_photon_orbit, L.ref_retrograde_photon_orbit):
        f.argtypes = [d]
        f.restype = d
    return L


def test_photon_sphere_golden_cases(an):
    """analytic_geodesic_reproducibility_test.cpp tests 1-9."""
    assert abs(an.radial_potential(3.0, 0.0, 0.0, 27.0)) < 1e-12
    assert an.critical_impact_params(3.0, 0.0) == (0.0, 27.0)
    a = 0.5
    r_ph = an.prograde_photon_orbit(a)
    xi, eta = an.critical_impact_params(r_ph, a)
    assert abs(an.radial_potential(r_ph, a, xi, eta)) < 1e-8
    assert an.radial_potential(2.0, 0.0, 0.0, 27.0) > 0 and an.radial_potential(5.0, 0.0, 0.0, 27.0) > 0
    assert abs(an.prograde_photon_orbit(0.0) - 3.0) < 1e-12
    assert abs(an.retrograde_photon_orbit(0.0) - 3.0) < 1e-12
    assert abs(an.prograde_photon_orbit(1.0) - 1.0) < 1e-12
    assert abs(an.retrograde_photon_orbit(1.0) - 4.0) < 1e-12
    pro = [an.prograde_photon_orbit(s) for s in (0.0, 0.5, 1.0)]
    ret = [an.retrograde_photon_orbit(s) for s in (0.0, 0.5, 1.0)]
    assert pro[0] > pro[1] > pro[2] and ret[0] < ret[1] < ret[2]
    # cuda_analytic_kerr_test.cu:201-218
    assert abs(an.prograde_photon_orbit(0.9) - 2.0 * (1.0 + math.cos(2.0 / 3.0 * math.acos(-0.9)))) < 1e-14


def test_quartic_roots_golden_round_trip(an, ref):
    """cuda_analytic_kerr_test.cu:224-267: r^4 - 35 r^2 + 90 r - 56 has roots
    4, 2, 1, -7; r(lambda0) = r3 and r(lambda0 + T/2) = r2 in the band between
    them. The reference's CPU findRadialRoots finds no real root here (its
    resolvent's 4/3 where the device version has 8/3)."""
    roots, n, motion = an.radial_roots(-35.0, 90.0, -56.0)
    assert n == 4 and motion == "transit"
    np.testing.assert_allclose(roots.real, [4.0, 2.0, 1.0, -7.0], rtol=0, atol=1e-13)
    assert np.all(roots.imag == 0.0)
    T2 = an.radial_half_period(roots.real)
    assert T2 > 0
    assert abs(an.r_bound(0.0, roots.real) - 1.0) < 1e-13
    assert abs(an.r_bound(T2, roots.real) - 2.0) < 1e-12
    assert abs(an.r_bound(2 * T2, roots.real) - 1.0) < 1e-12
    re, im, t = np.zeros(4), np.zeros(4), C.c_int()
    assert ref.ref_radial_roots(-35.0, 90.0, -56.0, re.ctypes.data, im.ctypes.data, C.byref(t)) == 0


def test_bound_motion_is_the_quadrature_inverse(an):
    """lambda(r) = int_r3^r dr / sqrt(R) inverts r_bound over the band."""
    rng = np.random.default_rng(5)
    for _ in range(20):
        r = rng.uniform(-3.0, 6.0, 3)
        roots = np.sort(np.append(r, -r.sum()))[::-1]
        R = lambda x: np.prod(x - roots)  # noqa: E731
        for f in (0.1, 0.5, 0.9):
            rt = roots[2] + f * (roots[1] - roots[2])
            lam = integrate.quad(lambda x: 1.0 / math.sqrt(R(x)), roots[2], rt, limit=200, epsabs=1e-13)[0]
            assert abs(an.r_bound(lam, roots) - rt) < 1e-9 * max(1.0, abs(rt))


def test_roots_against_numpy(an):
    rng = np.random.default_rng(2)
    for _ in range(300):
        a, xi, eta = rng.uniform(0, 0.999), rng.uniform(-8, 8), rng.uniform(-2, 40)
        c2, c1, c0 = an.quartic_coeffs(a, xi, eta)
        roots, n, _ = an.radial_roots(c2, c1, c0)
        want = np.roots([1.0, 0.0, c2, c1, c0])
        assert n == int(np.sum(np.abs(want.imag) < 1e-9 * np.maximum(1, np.abs(want))))
        np.testing.assert_allclose(np.sort_complex(roots), np.sort_complex(want),
                                   atol=1e-8 * max(1.0, np.abs(want).max()))
        for r in roots[:n].real:
            assert abs(an.radial_potential(r, a, xi, eta)) < 1e-9 * max(1.0, r ** 4)


def test_helpers_match_reference_build(an, ref):
    rng = np.random.default_rng(3)
    out = np.zeros(3)
    for _ in range(200):
        r, a, xi, eta = rng.uniform(1.0, 50.0), rng.uniform(-0.999, 0.999), rng.uniform(-10, 10), rng.uniform(-5, 50)
        assert an.radial_potential(r, a, xi, eta) == pytest.approx(ref.ref_radial_potential(r, a, xi, eta),
                                                                    rel=1e-13, abs=1e-9)
        ref.ref_quartic_coeffs(a, xi, eta, out.ctypes.data)
        np.testing.assert_allclose(an.quartic_coeffs(a, xi, eta), out, rtol=1e-13, atol=1e-12)
        r_ph = rng.uniform(1.01, 4.0)
        ref.ref_critical_impact_params(r_ph, a, out.ctypes.data)
        np.testing.assert_allclose(an.critical_impact_params(r_ph, a), out[:2], rtol=1e-13, atol=1e-12)
        assert an.prograde_photon_orbit(a) == pytest.approx(ref.ref_prograde_photon_orbit(a), rel=1e-15)
        assert an.retrograde_photon_orbit(a) == pytest.approx(ref.ref_retrograde_photon_orbit(a), rel=1e-15)


def test_jacobi_functions(an):
    """cuda_analytic_kerr_test.cu:136-196 cases, then any m <= 1 against mpmath."""
    assert an.ellpj(0.0, 0.25) == (0.0, 1.0, 1.0)
    sn, cn, dn = an.ellpj(1.0, 1e-4)
    assert abs(sn - math.sin(1.0)) < 2e-4 and abs(cn - math.cos(1.0)) < 2e-4 and abs(dn - 1.0) < 2e-4
    K = an.ellint_k(0.5)
    sn, cn, dn = an.ellpj(K, 0.25)
    assert abs(sn - 1.0) < 1e-14 and abs(cn) < 1e-14 and abs(dn - math.sqrt(0.75)) < 1e-14
    assert an.ellint_k(0.0) == pytest.approx(math.pi / 2, rel=1e-15)
    assert an.ellint_k(1.0) == math.inf
    mp.mp.dps = 30
    rng = np.random.default_rng(4)
    for _ in range(300):
        m = float(rng.choice([1.0 - 10 ** rng.uniform(-12, 0), -10 ** rng.uniform(-3, 1.5), rng.uniform(0, 1)]))
        u = rng.uniform(-12, 12)
        got = an.ellpj(u, m)
        want = [float(mp.re(mp.ellipfun(f, mp.mpf(u), m=mp.mpf(m)))) for f in ("sn", "cn", "dn")]
        np.testing.assert_allclose(got, want, rtol=0, atol=5e-13)
    for k in rng.uniform(0, 0.999999, 50):
        assert an.ellint_k(k) == pytest.approx(sp.ellipk(k * k), rel=1e-14)
    sn, cn, dn = an.ellpj(0.7, 1.0)
    assert (sn, cn, dn) == pytest.approx((math.tanh(0.7), 1 / math.cosh(0.7), 1 / math.cosh(0.7)), rel=1e-15)
