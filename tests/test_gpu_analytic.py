"""The closed-form image tracer (BH_INTEGRATOR_ANALYTIC, kerr_analytic.cuh) on
the GPU against the CPU oracle's FP64 DP45 at tight tolerances
(kerr_oracle.hpp): classes, disk radii, redshifts, fluxes and azimuths of every
crossing, escape directions, the near-critical band where the ray circles the
hole several times, the integrator fallback for rays the closed form leaves
out, the no-allocation entry point and the sky."""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np
import pytest
import torch

from blackhole_b200 import _abi, kerr

pytestmark = pytest.mark.gpu

ANALYTIC = _abi.INTEGRATOR_ANALYTIC


def _scene(n=48, spin=0.9, incl=60.0, form=1, maxc=3, **kw):
    s = _abi.default_scene(width=n, height=n, spin=spin, theta_obs=math.radians(incl), integrator=1,
                           max_crossings=maxc, precision=0)
    s.potential_form = form
    s.rtol, s.atol = 1e-11, 1e-13
    s.max_steps = 400000
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def _gpu(s, integrator=ANALYTIC, precision=0):
    g = _abi.KerrScene.from_buffer_copy(s)
    g.integrator = integrator
    g.precision = precision
    out = kerr.trace_image(g)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


def _wrap(x):
    return np.abs(np.angle(np.exp(1j * x)))


def _compare(got, ref, maxc, r_tol=1e-8, ang_tol=1e-8, inf_tol=1e-2, polar=None):
    """``polar``: pixels whose rays pass over the pole (angular momentum
    |lambda| ~ 1e-15 on an image column through alpha = 0). Passing the pole
    at an angular distance ~|lambda| turns the azimuth by pi within a Mino-time
    width ~|lambda|: the closed form has that turn, the oracle's stepper
    steps over it, so there phi is compared modulo pi."""
    ok = ref["cls"] != 3
    same = ok & (got["cls"] == ref["cls"])
    assert same.sum() >= 0.999 * ok.sum(), (same.sum(), ok.sum())
    np.testing.assert_array_equal(got["n_cross"][same], ref["n_cross"][same])
    for k in range(maxc):
        m = same & (ref["n_cross"] > k)
        if not m.any():
            continue
        np.testing.assert_allclose(got["r_hit"][k][m], ref["r_hit"][k][m], rtol=r_tol)
        np.testing.assert_allclose(got["g"][k][m], ref["g"][k][m], rtol=r_tol)
        dphi = _wrap(got["phi_hit"][k][m] - ref["phi_hit"][k][m])
        if polar is not None:
            dphi = np.where(polar[m], np.minimum(dphi, np.abs(dphi - np.pi)), dphi)
        assert dphi.max() < ang_tol
    hit = same & (ref["n_cross"] > 0)
    # absolute floor at r_tol of the frame's peak: the flux vanishes at the ISCO,
    # where its relative error is r's times r / (r - r_isco)
    for f, m in (("flux", hit), ("intensity", same)):
        np.testing.assert_allclose(got[f][m], ref[f][m], rtol=r_tol, atol=r_tol * np.abs(ref[f][m]).max(initial=0.0))
    esc = same & (ref["cls"] == 2)
    if esc.any():
        assert np.abs(got["theta_inf"][esc] - ref["theta_inf"][esc]).max() < inf_tol
        dinf = _wrap(got["phi_inf"][esc] - ref["phi_inf"][esc])
        if polar is not None:
            dinf = np.where(polar[esc], np.minimum(dinf, np.abs(dinf - np.pi)), dinf)
        assert dinf.max() < inf_tol
    assert np.all(got["steps"][same & (got["steps"] == 0)] == 0)
    return same


@pytest.mark.parametrize("spin,incl,form", [(0.9, 60.0, 1), (0.5, 80.0, 0), (0.99, 17.0, 1), (0.0, 45.0, 1),
                                            (0.9, 120.0, 1), (0.5, 150.0, 0)])
def test_analytic_matches_oracle(cuda, oracle, spin, incl, form):
    """Observers above and below the equator (120 and 150 deg: the polar
    motion starts at cos theta_obs < 0)."""
    s = _scene(spin=spin, incl=incl, form=form)
    got = _gpu(s)
    ref = oracle.trace_pixels(s)
    same = _compare(got, ref, 3)
    assert (got["steps"] == 0).mean() > 0.99  # all but the fallback pixels solved in closed form
    assert (ref["n_cross"][same] >= 2).any()


@pytest.mark.parametrize("spin,incl", [(0.998, 89.0), (-0.7, 30.0)])
def test_analytic_extreme_observers(cuda, oracle, spin, incl):
    """Near-extremal spin seen almost edge-on (the observer next to the
    equator, where the polar motion starts close to its crossing), and a
    retrograde hole, on a ragged 37 x 19 frame. Its middle column has
    |alpha| ~ 1e-15: those rays pass within ~1e-16 rad of the pole (see
    _compare); modulo that turn the closed form agrees with the oracle to
    ~1e-11 there as elsewhere."""
    s = _scene(spin=spin, incl=incl, width=37, height=19)
    got = _gpu(s)
    ref = oracle.trace_pixels(s)
    alpha = s.alpha_min + (np.arange(37 * 19) % 37 + 0.5) * (s.alpha_max - s.alpha_min) / 37
    _compare(got, ref, 3, polar=np.abs(alpha) < 1e-9)
    assert (got["steps"] == 0).mean() > 0.95


def test_analytic_pole_passing_rays(cuda, oracle):
    """Columns at alpha = +-1e-3 (|lambda| ~ 9e-4, 1 - z+ ~ 1e-8): those rays
    pass the pole at an angular distance the oracle's DP45 (rtol 1e-11)
    resolves, so it follows the azimuth's turn by pi and phi is compared
    without any modulo-pi relaxation. (Closer to the pole the steppers cannot
    follow: their right-hand side floors sin^2 theta at 1e-12, so a ray with
    1 - z+ below that -- alpha = 1e-5 here gives 9e-13 -- gets only part of
    the turn; the closed form's polar integral there agrees with a 50-digit
    quadrature.) The column at alpha = +0 (lambda = -0) gets the limit of the
    lambda < 0 side, a turn by copysign(pi, lambda) per pass over the pole:
    the same outputs as the column at alpha = 1e-12 to 1e-9."""
    for a0 in (1e-3, -1e-3):
        s = _scene(width=1, height=48, alpha_min=a0 - 0.5, alpha_max=a0 + 0.5)
        # the stepper's own error passing the pole there is ~3e-7 rad; a missing turn would be pi
        _compare(_gpu(s), oracle.trace_pixels(s), 3, ang_tol=1e-6)
    z = _gpu(_scene(width=1, height=48, alpha_min=-0.5, alpha_max=0.5))  # alpha = +0 exactly
    e = _gpu(_scene(width=1, height=48, alpha_min=1e-12 - 0.5, alpha_max=1e-12 + 0.5))
    np.testing.assert_array_equal(z["cls"], e["cls"])
    np.testing.assert_array_equal(z["n_cross"], e["n_cross"])
    assert (z["n_cross"] > 0).sum() >= 10 and (z["cls"] == 2).sum() >= 4
    for f in ("r_hit", "phi_hit", "g"):
        np.testing.assert_allclose(z[f], e[f], rtol=0, atol=1e-9, err_msg=f)
    for f in ("theta_inf", "phi_inf"):
        np.testing.assert_allclose(z[f], e[f], rtol=0, atol=1e-9, err_msg=f)


def test_analytic_single_pixel_and_partial_outputs(cuda, oracle):
    """A 1 x 1 frame through the image centre's neighbour, and a frame that
    asks for a subset of the outputs (the others NULL): the fields given are
    the full trace's, bit for bit."""
    one = _scene(n=1, alpha_min=-3.0, alpha_max=-2.9, beta_min=0.4, beta_max=0.5)
    got = _gpu(one)
    ref = oracle.trace_pixels(one)
    _compare(got, ref, 3)
    s = _abi.KerrScene.from_buffer_copy(_scene(n=40))
    s.integrator = ANALYTIC
    full = kerr.trace_image(s)
    part = {"cls": torch.full((1600,), -7, dtype=torch.int32, device="cuda"),
            "g": torch.full((3, 1600), -7.0, dtype=torch.float64, device="cuda")}
    kerr.trace_image(s, part)
    torch.cuda.synchronize()
    assert torch.equal(part["cls"], full["cls"])
    hit = full["n_cross"] > 0
    assert torch.equal(part["g"][0][hit], full["g"][0][hit])


def test_analytic_escape_direction_at_escape_radius(cuda, oracle):
    """The stepper reports the escape angles after its last step's overshoot
    past the escape radius (~1e-4 rad at 1.01 r_obs, up to ~3e-3 in phi next
    to the pole); with the escape radius far out that no longer shows and the
    angles agree to its integration error."""
    s = _scene(n=32, escape_factor=100.0)
    got = _gpu(s)
    ref = oracle.trace_pixels(s)
    _compare(got, ref, 3, inf_tol=5e-5)


def _critical_row(cuda_scene, n, half_width):
    """A one-row window across the shadow's edge on beta = 0 (retrograde
    side), located by bisection on the analytic tracer's class with the disk
    removed (escaped vs captured)."""
    lo, hi = 0.0, 12.0  # alpha: captured at 0, escapes at 12
    for _ in range(52):
        mid = 0.5 * (lo + hi)
        s = _abi.KerrScene.from_buffer_copy(cuda_scene)
        s.width, s.height = 1, 1
        s.alpha_min, s.alpha_max = mid - 1e-13, mid + 1e-13
        s.beta_min, s.beta_max = -1e-13, 1e-13
        s.disk_r_out = 1e-9
        c = _gpu(s)["cls"][0]
        if c == 2:
            hi = mid
        else:
            lo = mid
    s = _abi.KerrScene.from_buffer_copy(cuda_scene)
    s.width, s.height = n, 1
    s.alpha_min, s.alpha_max = lo - half_width, lo + half_width
    s.beta_min, s.beta_max = -1e-9, 1e-9
    return s


def test_analytic_near_critical_band(cuda, oracle):
    """Rays within 1e-6 M of the shadow's edge (1 - m ~ 1e-8) circle the hole
    and cross the disk plane several times; the closed form agrees with the
    long-double oracle (whose own error there is ~5e-12 in r against a
    40-digit evaluation of the same closed form)."""
    base = _scene(spin=0.9, incl=80.0, form=1, maxc=3, disk_r_out=60.0)
    s = _critical_row(base, 64, 1e-6)
    got = _gpu(s)
    alpha = s.alpha_min + (np.arange(64) + 0.5) * (s.alpha_max - s.alpha_min) / 64
    ref = oracle.trace_alpha_beta(s, alpha, np.zeros(64), long_double=True)
    assert (got["n_cross"] >= 2).sum() >= 32
    assert (got["steps"] == 0).all()
    _compare(got, ref, 3, r_tol=1e-9, ang_tol=1e-7)


def test_analytic_fallback_pixels_are_stepped(cuda, oracle):
    """A ray whose turning point lies between r+ and the horizon cut (here
    1.5 r+, next to the prograde edge of the shadow) is left to DP45, whose
    outputs it carries (steps > 0), at both precisions."""
    s = _scene(n=64, spin=0.9, incl=80.0, form=1, horizon_factor=1.5, alpha_min=-8.0, alpha_max=8.0,
               beta_min=-8.0, beta_max=8.0)
    ref = oracle.trace_pixels(s)
    for prec in (0, 1):
        got = _gpu(s, precision=prec)
        stepped = got["steps"] > 0
        assert stepped.any() and stepped.mean() < 0.5
        dp = _gpu(s, integrator=1, precision=prec)
        for k in ("cls", "n_cross", "steps"):
            np.testing.assert_array_equal(got[k][stepped], dp[k][stepped])
        np.testing.assert_array_equal(got["theta_inf"][stepped], dp["theta_inf"][stepped])
        _compare(got, ref, 3, r_tol=1e-8 if prec == 0 else 1e-5, ang_tol=1e-8 if prec == 0 else 1e-3)


def test_analytic_no_allocation_entry(cuda, oracle):
    """bh_kerr_trace_image_host_noalloc keeps the fallback list in its fixed
    scratch: same outputs as the allocating host entry point."""
    s = _scene(n=64, spin=0.9, incl=80.0, form=1, horizon_factor=1.5, alpha_min=-8.0, alpha_max=8.0,
               beta_min=-8.0, beta_max=8.0)
    s.integrator = ANALYTIC
    fields = ("cls", "steps", "n_cross", "r_hit", "g", "phi_hit", "theta_inf")
    a = kerr.trace_image_host(s, fields)
    b = kerr.trace_image_host_noalloc(s, fields)
    assert (a["steps"] > 0).any()
    for k in fields:
        np.testing.assert_array_equal(a[k], b[k])


def test_analytic_sky_radiance(cuda, oracle):
    """Escaped rays add the cubemap's radiance in their direction of motion at
    the escape radius; with the escape radius far out the texel is the one
    the stepper reads for nearly every pixel."""
    sky = kerr.sky_generate(64, seed=7, n_stars=2000)
    s = _scene(n=48, escape_factor=100.0, maxc=1, disk_r_out=8.0, alpha_min=-20.0, alpha_max=20.0,
               beta_min=-20.0, beta_max=20.0)
    g = _abi.KerrScene.from_buffer_copy(s)
    g.integrator = ANALYTIC
    got = {k: v.cpu().numpy() for k, v in kerr.trace_image(g, sky=sky).items()}
    d = _abi.KerrScene.from_buffer_copy(s)
    d.integrator = 1
    dp = {k: v.cpu().numpy() for k, v in kerr.trace_image(d, sky=sky).items()}
    torch.cuda.synchronize()
    esc = (got["cls"] == 2) & (dp["cls"] == 2)
    assert esc.mean() > 0.3
    same = np.isclose(got["intensity"][esc], dp["intensity"][esc], rtol=1e-9)
    assert same.mean() >= 0.98


REF_DEV = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libbh_ref_analytic_dev.so"


@pytest.mark.skipif(not REF_DEV.exists(), reason="reference device build absent (oracle/_ref)")
def test_helpers_match_reference_device_functions(cuda):
    """include/bh_analytic.h (FP64, host) against the reference's own FP32
    device helpers (src/cuda/device_analytic_kerr.cuh, compiled unmodified):
    d_ellpj, d_ellint_K, d_quartic_real_roots, d_kerr_r_analytic,
    d_kerr_radial_half_period and the photon orbits, at FP32 tolerances."""
    from blackhole_b200 import analytic as an

    L = C.CDLL(str(REF_DEV))
    vp, i = C.c_void_p, C.c_int
    for name, args in (("ref_dev_ellpj", [i, vp, vp, vp]), ("ref_dev_ellint_k", [i, vp, vp]),
                       ("ref_dev_roots", [i, vp, vp]), ("ref_dev_r_analytic", [i, vp, vp, C.c_float, vp]),
                       ("ref_dev_half_period", [i, vp, vp]), ("ref_dev_critical", [i, vp, vp, vp]),
                       ("ref_dev_photon", [i, vp, vp])):
        getattr(L, name).argtypes = args
    f32 = lambda x: np.ascontiguousarray(x, np.float32)  # noqa: E731
    rng = np.random.default_rng(11)
    n = 256
    u, m = f32(rng.uniform(-8, 8, n)), f32(rng.uniform(1e-4, 0.98, n))
    out = np.zeros(3 * n, np.float32)
    assert L.ref_dev_ellpj(n, u.ctypes.data, m.ctypes.data, out.ctypes.data) == 0
    ours = np.array([an.ellpj(float(a), float(b)) for a, b in zip(u, m)]).ravel()
    np.testing.assert_allclose(ours, out, atol=2e-4)
    k = f32(rng.uniform(0, 0.99, n))
    out = np.zeros(n, np.float32)
    assert L.ref_dev_ellint_k(n, k.ctypes.data, out.ctypes.data) == 0
    np.testing.assert_allclose([an.ellint_k(float(x)) for x in k], out, rtol=1e-5)
    # quartics with four well-separated real roots summing to zero, descending
    r3 = rng.uniform(-3, 6, (n, 3))
    roots = np.sort(np.concatenate([r3, -r3.sum(1, keepdims=True)], 1), axis=1)[:, ::-1]
    roots = roots[np.min(-np.diff(roots, axis=1), axis=1) > 0.3][:64]
    nq = len(roots)
    c = np.stack([np.poly(r)[2:] for r in roots])
    out = np.zeros(5 * nq, np.float32)
    assert L.ref_dev_roots(nq, f32(c).ctypes.data, out.ctypes.data) == 0
    out = out.reshape(nq, 5)
    for q in range(nq):
        got, nr, _ = an.radial_roots(*c[q])
        assert nr == int(out[q, 0]) == 4
        np.testing.assert_allclose(got.real, out[q, 1:], atol=2e-3 * max(1.0, np.abs(roots[q]).max()))
    lam = f32(rng.uniform(0, 3, nq))
    ro = f32(roots)
    out = np.zeros(nq, np.float32)
    assert L.ref_dev_r_analytic(nq, lam.ctypes.data, ro.ctypes.data, 0.0, out.ctypes.data) == 0
    np.testing.assert_allclose([an.r_bound(float(x), r) for x, r in zip(lam, roots)], out, rtol=2e-4, atol=2e-4)
    assert L.ref_dev_half_period(nq, ro.ctypes.data, out.ctypes.data) == 0
    np.testing.assert_allclose([an.radial_half_period(r) for r in roots], out, rtol=2e-5)
    # d_critical_impact_params (device_analytic_kerr.cuh:418-449) has 2 r Delta / (a Delta')
    # in xi and drops a factor r from eta; ours is Bardeen's xi, eta as in the reference's
    # CPU criticalImpactParams (pinned in tests/test_analytic_api.py): R = 0 there, not at the device's.
    rph, a = f32(rng.uniform(1.2, 4.0, n)), f32(rng.uniform(0.05, 0.99, n))
    out = np.zeros(2 * n, np.float32)
    assert L.ref_dev_critical(n, rph.ctypes.data, a.ctypes.data, out.ctypes.data) == 0
    r_dev = []
    for r, s, dev in zip(rph[:16], a[:16], out.reshape(n, 2)[:16]):
        xi, eta = an.critical_impact_params(float(r), float(s))
        assert abs(an.radial_potential(float(r), float(s), xi, eta)) < 1e-9 * float(r) ** 4
        r_dev.append(abs(an.radial_potential(float(r), float(s), float(dev[0]), float(dev[1]))))
    assert max(r_dev) > 1e-2
    assert L.ref_dev_photon(n, a.ctypes.data, out.ctypes.data) == 0
    ours = np.array([(an.prograde_photon_orbit(float(s)), an.retrograde_photon_orbit(float(s))) for s in a]).ravel()
    np.testing.assert_allclose(ours, out, rtol=1e-5)
