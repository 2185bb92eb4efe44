"""GPU checks of the surrogate renderer (bh_surrogate_trace_image).

* with an untrained network no pixel is confident, so every pixel goes to
  the renderer's fallback, the closed-form tracer (DP45 on the rays it does
  not cover): the image equals that tracer's bit for bit;
* with the confidence gate off and the solved class final (verify 3: an
  untrained network only seeds the solve), every pixel the exact solve
  decides matches the FP64 oracle: class, disk radius, redshift, flux and
  the azimuth of the hit; escape directions match the closed-form tracer,
  which is exact at the escape radius; observers above and below the
  equator;
* with the trained network shipped in blackhole_b200/data, the a = 0.9
  disk scene meets the accuracy targets on every output field;
* rays on the image column through alpha = 0 (lambda = -0) pass over the
  pole: the solve applies the same turn by pi as the closed-form tracer;
* ablation at equal outputs: what the trained network gains over the same
  renderer without it.
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

WEIGHTS = Path(__file__).resolve().parent.parent / "blackhole_b200" / "data" / "surrogate_c4.npz"
ALL_FIELDS = ("cls", "steps", "n_cross", "r_hit", "phi_hit", "g", "flux", "intensity", "theta_inf", "phi_inf")
DISK_FIELDS = tuple(f for f in ALL_FIELDS if f not in ("phi_hit", "phi_inf"))

# Stated error bounds of an accepted pixel against the FP64 references
# (FP32 quadrature and elliptic integrals by default; all FP64 on request):
# r and g relative (r: p99.9 and max), azimuths and theta_inf in radians
# (modulo 2 pi). The FP32 solve's worst pixels are rays whose radial turning
# point lies just outside the critical band, next to the photon orbit, where
# the radial integral is nearly singular (5e-5 on a 77 x 53 frame).
TOL = {False: dict(r=2e-5, r_max=1e-4, ang=5e-5, theta=2e-6),
       True: dict(r=1e-6, r_max=1e-6, ang=1e-6, theta=1e-7)}


def c4_scene(W, **kw):
    from blackhole_b200 import kerr

    args = dict(width=W, height=W, spin=0.9, theta_obs=math.radians(60), integrator=1, max_crossings=1)
    args.update(kw)
    return kerr.scene(**args)


def host(o):
    return {k: v.cpu().numpy() for k, v in o.items()}


def wrap(x):
    return np.abs(np.angle(np.exp(1j * x)))


def pole_column(s):
    """Pixels whose image-plane alpha is zero to rounding (the middle column
    of an odd-width frame): their rays pass within ~|lambda| of the pole,
    where the azimuth turns by pi in a Mino-time width ~|lambda| that the
    oracle's stepper steps over, so their azimuths are compared modulo pi."""
    i = np.arange(s.width)
    da = (s.alpha_max - s.alpha_min) / s.width
    alpha = s.alpha_min + (i + 0.5) * da
    col = np.abs(alpha) < 1e-9 * da
    return np.tile(col, s.height)


def wrap_pi(x):
    """|x| modulo pi, in [0, pi / 2]."""
    m = np.mod(np.abs(x), np.pi)
    return np.minimum(m, np.pi - m)


def closed_form(s):
    """The closed-form FP64 tracer on the same frame (all fields)."""
    from blackhole_b200 import _abi, kerr

    sa = _abi.KerrScene.from_buffer_copy(s)
    sa.integrator = _abi.INTEGRATOR_ANALYTIC
    sa.precision = 0
    out = host(kerr.trace_image(sa))
    torch.cuda.synchronize()
    return out


def test_untrained_network_falls_back_everywhere(cuda):
    from blackhole_b200 import _abi, kerr
    from blackhole_b200 import surrogate as S

    net = S.Surrogate(max_batch=128, seed=3)
    s = c4_scene(96, precision=1)
    got = host(net.trace_image(s))
    st = net.last_stats()
    assert st["pixels"] == 96 * 96 and st["accepted"] == 0 and st["low_confidence"] == 96 * 96
    sa = _abi.KerrScene.from_buffer_copy(s)
    sa.integrator = _abi.INTEGRATOR_ANALYTIC
    ref = host(kerr.trace_image(sa))
    torch.cuda.synchronize()
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


@pytest.mark.parametrize("fp64", [True, False])
@pytest.mark.parametrize("spin,incl,form", [(0.9, 60, 0), (0.998, 85, 0), (0.3, 17, 1), (0.7, 125, 0)])
def test_exact_solve_matches_oracle(cuda, oracle, spin, incl, form, fp64):
    _check_exact_solve(oracle, spin, incl, form, fp64, 80, 80)


@pytest.mark.parametrize("fp64", [True, False])
def test_exact_solve_matches_oracle_ragged(cuda, oracle, fp64):
    """A 77 x 53 frame: its second chunk ends inside a CTA of the
    refinement, whose idle threads still pass the phase barriers."""
    _check_exact_solve(oracle, 0.9, 60, 0, fp64, 77, 53)


def _check_exact_solve(oracle, spin, incl, form, fp64, W, H):
    from blackhole_b200 import surrogate as S

    net = S.Surrogate(max_batch=128, seed=4)
    s = c4_scene(W, height=H, spin=spin, theta_obs=math.radians(incl), potential_form=form, precision=1)
    got = host(net.trace_image(s, min_confidence=0.0, verify=3, critical_band=0.05, refine_fp64=fp64))
    tol = TOL[fp64]
    st = net.last_stats()
    # verify 3: the solve decides every pixel outside the critical band (the network only seeds it)
    assert st["accepted"] > 0.9 * st["pixels"] and st["solve_failed"] < 0.01 * st["pixels"], st
    so = c4_scene(W, height=H, spin=spin, theta_obs=math.radians(incl), potential_form=form, precision=0)
    ref = oracle.trace_pixels(so)
    acc = got["steps"] == 0  # answered without the integrator
    np.testing.assert_array_equal(got["cls"][acc], ref["cls"][acc])
    assert np.mean(got["cls"] == ref["cls"]) >= 0.999
    d = acc & (ref["n_cross"] > 0)
    assert d.any()
    for f in ("r_hit", "g"):
        rel = np.abs(got[f][0][d] - ref[f][0][d]) / np.abs(ref[f][0][d])
        assert np.quantile(rel, 0.999) <= tol["r"] and rel.max() <= tol["r_max"], (f, np.quantile(rel, 0.999), rel.max())
    # NT flux ~ (1 - sqrt(r_isco / r)) / r^3 amplifies a radius error next to the ISCO
    np.testing.assert_allclose(got["flux"][d], ref["flux"][d], rtol=10 * tol["r_max"], atol=1e-6)
    # the oracle's DP45 (rtol 1e-8) carries ~1e-8 of its own in the azimuth
    pole = pole_column(s)
    dphi = np.where(pole, wrap_pi(got["phi_hit"][0] - ref["phi_hit"][0]), wrap(got["phi_hit"][0] - ref["phi_hit"][0]))
    assert dphi[d].max() < tol["ang"] + 1e-7
    # escape angles against the closed form, which is exact at the escape radius
    cf = closed_form(so)
    esc = acc & (ref["cls"] == 2) & (cf["cls"] == 2)
    assert esc.any()
    assert np.abs(got["theta_inf"][esc] - cf["theta_inf"][esc]).max() < tol["theta"]
    assert wrap(got["phi_inf"][esc] - cf["phi_inf"][esc]).max() < tol["ang"]
    # and against the oracle's stepper, whose last step overshoots the escape radius (~1e-4 rad)
    assert np.abs(got["theta_inf"][esc] - ref["theta_inf"][esc]).max() < 2e-3


@pytest.mark.parametrize("fp64", [True, False])
def test_pole_passing_rays_turn_like_the_closed_form(cuda, fp64):
    """1 x 1 frames on the column through alpha = +0 (lambda = -0: the ray
    goes over the pole) and at |alpha| = 1e-5 and 1e-12 beside it, above and
    below the shadow: the solve gives the closed-form tracer's azimuths,
    including its turn by pi at each pass over the pole (copysign(pi, lambda)
    at lambda = -0, so alpha = +0 continues the alpha > 0 side), and escape
    directions on a frame without a disk."""
    from blackhole_b200 import surrogate as S

    net = S.Surrogate(max_batch=128, seed=4)
    tol = TOL[fp64]

    def one(a0, beta, **kw):
        s = c4_scene(1, alpha_min=a0 - 1.0, alpha_max=a0 + 1.0, beta_min=beta - 0.5, beta_max=beta + 0.5,
                     precision=1, **kw)
        got = host(net.trace_image(s, min_confidence=0.0, verify=3, critical_band=0.0, refine_fp64=fp64))
        assert net.last_stats()["accepted"] == 1, (a0, beta, net.last_stats())
        return got, closed_form(s)

    for a0 in (0.0, 1e-5, -1e-5, 1e-12):
        for beta in (-6.0, 4.5, 7.0):
            got, cf = one(a0, beta)
            assert got["cls"][0] == cf["cls"][0] == 1, (a0, beta)
            assert wrap(got["phi_hit"][0] - cf["phi_hit"][0]).max() < tol["ang"], (a0, beta)
            np.testing.assert_allclose(got["r_hit"][0], cf["r_hit"][0], rtol=tol["r"])
        for beta in (-9.0, 7.0):  # no disk: the ray escapes after passing over the pole
            got, cf = one(a0, beta, disk_r_out=1e-9)
            assert got["cls"][0] == cf["cls"][0] == 2, (a0, beta)
            assert wrap(got["phi_inf"] - cf["phi_inf"]).max() < tol["ang"], (a0, beta)
            assert np.abs(got["theta_inf"] - cf["theta_inf"]).max() < tol["theta"], (a0, beta)
    # alpha = +0 against alpha = 1e-12 (lambda -> 0 from below): the same turn
    z, _ = one(0.0, 7.0)
    e, _ = one(1e-12, 7.0)
    assert abs(z["phi_hit"][0][0] - e["phi_hit"][0][0]) < 1e-6


def field_errors(got, ref, cf):
    """Per-field errors of ``got`` on pixels whose class agrees: against the
    FP64 DP45 tracer (class, r, g, phi_hit, flux, intensity) and the closed
    form (escape angles at the escape radius)."""
    same = got["cls"] == ref["cls"]
    d = same & (got["n_cross"] > 0) & (ref["n_cross"] > 0)
    esc = same & (ref["cls"] == 2) & (cf["cls"] == 2)
    fpk, ipk = np.abs(ref["flux"]).max(), np.abs(ref["intensity"]).max()
    return {
        "class": np.mean(same),
        "r": np.abs(got["r_hit"][0][d] - ref["r_hit"][0][d]) / ref["r_hit"][0][d],
        "g": np.abs(got["g"][0][d] - ref["g"][0][d]) / ref["g"][0][d],
        "phi_hit": wrap(got["phi_hit"][0][d] - ref["phi_hit"][0][d]),
        "flux": np.abs(got["flux"][d] - ref["flux"][d]) / fpk,
        "intensity": np.abs(got["intensity"][same] - ref["intensity"][same]) / ipk,
        "theta_inf": np.abs(got["theta_inf"][esc] - cf["theta_inf"][esc]),
        "phi_inf": wrap(got["phi_inf"][esc] - cf["phi_inf"][esc]),
    }


@pytest.mark.skipif(not WEIGHTS.exists(), reason="trained weights not shipped")
def test_trained_network_meets_targets(cuda):
    """The committed network on the 512^2 a = 0.9, 60 deg disk frame: class
    agreement >= 99.9 % and dg/g median <= 1e-4, max <= 1e-3 against the FP64
    DP45 tracer (the targets), and stated bounds on every other output."""
    from blackhole_b200 import kerr
    from blackhole_b200 import surrogate as S

    net = S.Surrogate(max_batch=128)
    net.load(WEIGHTS)
    s = c4_scene(512, precision=1)
    outs = kerr.alloc_image_outputs(s, fields=list(ALL_FIELDS))
    got = host(net.trace_image(s, outs))
    st = net.last_stats()
    assert st["accepted"] > 0.95 * st["pixels"], st
    s64 = c4_scene(512, precision=0)
    ref = host(kerr.trace_image(s64, kerr.alloc_image_outputs(s64, fields=list(ALL_FIELDS))))
    cf = closed_form(s64)
    e = field_errors(got, ref, cf)
    assert e["class"] >= 0.999, e["class"]
    assert np.median(e["g"]) <= 1e-4 and e["g"].max() <= 1e-3, (np.median(e["g"]), e["g"].max())
    # stated bounds (the FP32 solve; the DP45 reference carries ~1e-8 of its own)
    assert e["r"].max() <= 1e-4 and np.median(e["r"]) <= 1e-6, (np.median(e["r"]), e["r"].max())
    assert e["g"].max() <= 1e-4
    assert e["flux"].max() <= 1e-4 and e["intensity"].max() <= 1e-4, (e["flux"].max(), e["intensity"].max())
    assert e["phi_hit"].max() <= 1e-3 and np.median(e["phi_hit"]) <= 1e-5, \
        (np.median(e["phi_hit"]), e["phi_hit"].max())
    assert e["theta_inf"].max() <= 1e-4 and e["phi_inf"].max() <= 1e-3, (e["theta_inf"].max(), e["phi_inf"].max())
    assert np.median(e["phi_inf"]) <= 1e-5


def _ms(fn, reps=5):
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        fn()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


@pytest.mark.skipif(not WEIGHTS.exists(), reason="trained weights not shipped")
def test_trained_network_gain_at_equal_outputs(cuda):
    """Ablation at equal outputs and equal accuracy. The method without the
    network is the same renderer with an untrained network: every pixel goes
    to its fallback, the closed-form tracer, and every field comes from an
    exact solve either way. With every field (azimuths included) the trained
    network must be faster than that fallback and >= 1.5x faster than the
    mixed DP45 tracer, taking none of its steps beyond 5 %. With the disk
    fields only (no azimuths) the closed form alone is the faster method;
    the test records that instead of asserting a gain."""
    from blackhole_b200 import _abi, kerr
    from blackhole_b200 import surrogate as S

    s = c4_scene(1024, precision=1)
    trained = S.Surrogate(max_batch=128)
    trained.load(WEIGHTS)
    blank = S.Surrogate(max_batch=128, seed=3)
    o_t = kerr.alloc_image_outputs(s, fields=list(ALL_FIELDS))
    o_b = kerr.alloc_image_outputs(s, fields=list(ALL_FIELDS))
    o_m = kerr.alloc_image_outputs(s, fields=list(ALL_FIELDS))
    trained.trace_image(s, o_t)
    blank.trace_image(s, o_b)
    kerr.trace_image(s, o_m)
    torch.cuda.synchronize()
    steps_t = int(o_t["steps"].sum().item())
    steps_m = int(o_m["steps"].sum().item())
    assert steps_t <= 0.05 * steps_m, (steps_t, steps_m)
    t_net = _ms(lambda: trained.trace_image(s, o_t))
    t_blank = _ms(lambda: blank.trace_image(s, o_b))
    t_plain = _ms(lambda: kerr.trace_image(s, o_m))
    assert t_plain >= 1.5 * t_net, (t_plain, t_net)
    assert t_blank > t_net, (t_blank, t_net)
    # disk fields only: recorded, not asserted (the closed form needs no network there)
    sa = _abi.KerrScene.from_buffer_copy(s)
    sa.integrator = _abi.INTEGRATOR_ANALYTIC
    sa.precision = 0
    o_d = kerr.alloc_image_outputs(s, fields=list(DISK_FIELDS))
    o_a = kerr.alloc_image_outputs(sa, fields=list(DISK_FIELDS))
    t_net_d = _ms(lambda: trained.trace_image(s, o_d))
    t_cf_d = _ms(lambda: kerr.trace_image(sa, o_a))
    print(f"\nall fields: trained {t_net:.3f} ms, fallback only {t_blank:.3f} ms, mixed DP45 {t_plain:.3f} ms; "
          f"disk fields: trained {t_net_d:.3f} ms, closed form {t_cf_d:.3f} ms")


def _host_render(net, s, pinned, chunks=0):
    """bh_surrogate_trace_image_host into pinned (torch) or pageable (numpy)
    buffers of every field."""
    import ctypes as C

    from blackhole_b200 import _abi

    n = s.width * s.height
    outs = {f: torch.zeros(n * (s.max_crossings if f in _abi.PLANE_FIELDS else 1),
                           dtype=torch.int32 if f in _abi.INT_FIELDS else torch.float64) for f in ALL_FIELDS}
    if pinned:
        outs = {f: t.pin_memory() for f, t in outs.items()}
    o = _abi.KerrImageOut()
    for f, t in outs.items():
        setattr(o, f, t.data_ptr())
    pol = _abi.SurrogatePolicy(0.99, 1, 0.05, 0, chunks)
    _abi.check(net._lib.bh_surrogate_trace_image_host(net._h, C.byref(s), C.byref(o), C.byref(pol)))
    return {f: t.numpy().reshape(-1) for f, t in outs.items()}


@pytest.mark.parametrize("trained,pinned,chunks,shape", [(True, True, 0, (320, 320, 1)), (True, True, 3, (320, 320, 1)),
                                                         (True, False, 0, (320, 320, 1)), (False, True, 0, (320, 320, 1)),
                                                         (False, False, 0, (320, 320, 1)), (True, True, 0, (333, 217, 3)),
                                                         (True, True, 5, (61, 47, 2)), (False, True, 0, (61, 47, 3))])
def test_host_buffers_match_device_render(cuda, trained, pinned, chunks, shape):
    """The host-buffer entry point returns the device render's outputs bit
    for bit. Pinned buffers take the overlapped path: each chunk's rows are
    copied while the next is inferred, and the rejected pixels follow in
    compact form (with one crossing plane the trained network rejects under
    1 %); with an untrained
    network every pixel is rejected, more than the compact buffers hold
    (except on frames of at most 4096 pixels, where the compact buffers hold
    the whole frame), and the frame is copied again. Pageable buffers are
    copied after the render. Ragged frames with two or three crossing planes
    check the per-plane row offsets."""
    from blackhole_b200 import kerr
    from blackhole_b200 import surrogate as S

    if trained and not WEIGHTS.exists():
        pytest.skip("trained weights not shipped")
    net = S.Surrogate(max_batch=128, seed=3)
    if trained:
        net.load(WEIGHTS)
    # Ragged sizes and several crossing planes exercise the per-plane row
    # copies. With more than one plane, rays that hit the disk once and escape
    # go to the integrator, so the 333 x 217 frame rejects more pixels than
    # the compact buffers hold (the frame is copied again), while frames of at
    # most 4096 pixels fit the compact buffers whole (gathered and scattered).
    W, H, mc = shape
    s = c4_scene(W, height=H, max_crossings=mc, precision=1)
    ref = host(net.trace_image(s, kerr.alloc_image_outputs(s, fields=list(ALL_FIELDS))))
    torch.cuda.synchronize()
    st = net.last_stats()
    rejected = st["pixels"] - st["accepted"]
    if mc == 1:
        assert (0 < rejected < 4096) if trained else rejected == st["pixels"], st
    else:
        assert rejected > 0, st
    for _ in range(2):  # the second call reuses the grown buffers
        got = _host_render(net, s, pinned, chunks)
        for f in ALL_FIELDS:
            np.testing.assert_array_equal(got[f], ref[f].reshape(-1), err_msg=f)
