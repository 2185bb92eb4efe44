"""The reference renderer's launch ABI on the GPU (include/bh_legacy.h), through
the C ABI: camera rays, shading, the backend, the Blender-bridge calls, the
lensing map, the disk texture and the geodesic paths, each against the CPU
oracle (kerr_oracle.hpp camera/paths, oracle/legacy_oracle.py shading)."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest
import torch

from oracle import legacy_oracle as LO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def leg():
    from blackhole_b200 import legacy

    legacy.library()
    return legacy


def _render(leg, p, variant=-1):
    fb = torch.zeros(p.height * p.width * 4, dtype=torch.float32, device="cuda")
    leg.launch(p, fb, variant)
    torch.cuda.synchronize()
    return fb.view(p.height * p.width, 4).cpu().numpy()


def _oracle_frame(oracle, p):
    kw, cf, ci = LO.camera(p)
    return oracle.trace_camera(LO.scene_of(kw), cf, ci), cf


@pytest.mark.parametrize("spin,r_rs,incl", [(0.9, 15.0, 1.3), (0.5, 40.0, 0.35), (0.0, 10.0, math.pi / 2)])
def test_camera_render_matches_oracle(cuda, leg, oracle, spin, r_rs, incl):
    p = leg.bridge_params(spin, r_rs, incl, 0.6, 64, 48)
    p.max_steps = 4000
    got = _render(leg, p)
    ref, cf = _oracle_frame(oracle, p)
    want = LO.shade(ref, p, cf[15], cf[16])
    hit = ref["cls"] == 1
    assert hit.any() and (ref["cls"] == 0).any()
    # classes are not an output here: a pixel that changed class changes colour wholesale
    lum = lambda x: x[:, :3].sum(1)  # noqa: E731
    same = (lum(got) > 0) == hit
    assert same.mean() >= 0.995, same.mean()
    both = same & hit
    np.testing.assert_allclose(got[both], want[both], rtol=2e-4, atol=1e-6)
    np.testing.assert_array_equal(got[~hit & same], np.array([[0, 0, 0, 1]] * int((~hit & same).sum()), np.float32))


def test_far_camera_sees_the_distant_observer_image(cuda, leg, oracle):
    """Orientation and scale of the camera model: a camera 2000 M away with a
    narrow field sees the image plane of a distant observer at its
    inclination to O(1/r), alpha = r u, beta = r v (u, v the pixel's
    image-plane offsets; the bridge camera's up vector points away from the
    projected spin axis, so rows run along +beta as in the image tracer) --
    its disk-hit map equals the image tracer's."""
    r_m, incl, n = 2000.0, 1.0, 48
    p = leg.bridge_params(0.7, r_m / 2, incl, 1.0, n, n)
    p.fov_scale = 12.0 / r_m  # the bridge clamps its field of view at 0.05; the launch ABI does not
    p.max_dist = 1.02 * r_m / 2
    p.max_steps = 20000
    got = _render(leg, p)
    cam_hit = (got[:, :3].sum(1) > 0).reshape(n, n)
    from blackhole_b200._abi import default_scene

    s = default_scene(width=n, height=n, spin=0.7, theta_obs=incl, integrator=1, max_crossings=1, precision=0)
    s.r_obs = r_m
    s.potential_form = 1
    s.disk_r_out = 60.0
    s.disk_r_in = 2.0 * float(p.isco)
    ref = oracle.trace_pixels(s)
    img_hit = (ref["cls"] == 1).reshape(n, n)
    assert 0.2 < img_hit.mean() < 0.95
    assert (cam_hit == img_hit).mean() >= 0.99, (cam_hit == img_hit).mean()


def test_backend_renders_the_same_frame(cuda, leg, lib):
    from cuda.bindings import runtime as rt

    L = leg.library()
    p = leg.bridge_params(0.9, 20.0, 1.2, 0.7, 40, 30)
    b = L.bhCudaInit(0, 40, 30)
    assert b
    try:
        assert L.bhCudaGetVariant(b) == -1
        assert L.bhCudaSetVariant(b, 2) == 2
        assert L.bhCudaSetVariant(b, 9) == -1
        assert L.bhCudaRegisterLut(b, 0, 7, 0x0DE1) == -1
        assert L.bhCudaRenderFrame(b, C.byref(p)) == 0
        host = np.zeros((30 * 40, 4), np.float32)
        err, = rt.cudaMemcpy(host.ctypes.data, L.bhCudaFramebuffer(b), host.nbytes,
                             rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
        assert int(err) == 0
        np.testing.assert_array_equal(host, _render(leg, p))
        bad = leg.bridge_params(0.9, 20.0, 1.2, 0.7, 41, 30)
        assert L.bhCudaRenderFrame(b, C.byref(bad)) == -1
        assert L.bhCudaResize(b, 0, 41, 30) == 0
        assert L.bhCudaRenderFrame(b, C.byref(bad)) == 0
    finally:
        L.bhCudaShutdown(b)


def test_bridge_render_is_tonemapped_shading(cuda, leg, oracle):
    spin, r_rs, incl, w, h = 0.8, 25.0, 1.25, 48, 36
    img = leg.render_raytraced(spin, r_rs, incl, w, h).reshape(-1, 4)
    p = leg.bridge_params(spin, r_rs, incl, 1.0, w, h)
    ref, cf = _oracle_frame(oracle, p)
    want = LO.shade(ref, p, cf[15], cf[16], exposure=12.0)
    assert np.all(img[:, 3] == 1.0) and img.min() >= 0.0 and img.max() <= 1.0
    same = (img[:, :3].sum(1) > 0) == (ref["cls"] == 1)
    assert same.mean() >= 0.99
    np.testing.assert_allclose(img[same], want[same], rtol=2e-4, atol=2e-6)
    alias = np.zeros((h, w, 4), np.float32)
    assert leg.library().bhb_cuda_render_raytraced(spin, r_rs, incl, w, h, alias.ctypes.data) == 0
    np.testing.assert_array_equal(alias.reshape(-1, 4), img)


def test_lensing_map_matches_oracle(cuda, leg, oracle):
    a, r_obs, incl, w, h = 0.9, 500.0, 1.1, 40, 32
    got = leg.lensing_map(a, r_obs, incl, w, h).reshape(-1, 4)
    from blackhole_b200._abi import default_scene

    s = default_scene(width=w, height=h, spin=a, theta_obs=incl, integrator=1, max_crossings=1, precision=0)
    s.r_obs = r_obs
    s.potential_form = 1
    s.disk_r_out = 100.0
    i, j = np.meshgrid(np.arange(w), np.arange(h))
    alpha = (30.0 * (i / w - 0.5)).ravel()
    beta = (30.0 * (0.5 - j / h)).ravel()
    ref = oracle.trace_alpha_beta(s, alpha, beta)
    want = LO.lensing(ref)
    same = got[:, 2] == want[:, 2]
    assert same.mean() >= 0.995
    np.testing.assert_allclose(got[same], want[same], rtol=1e-5, atol=1e-6)


def test_disk_texture_matches_restatement(cuda, leg):
    from blackhole_b200 import legacy

    a, r_out, incl, w, h = 0.6, 40.0, 1.0, 64, 32
    got = leg.disk_texture(a, r_out, incl, w, h)
    r_isco = legacy.isco_prograde(a)
    rp = 1.5 * r_isco
    peak = (1 - math.sqrt(r_isco / rp)) / rp ** 3
    want = LO.disk_texture(a, r_isco, r_out, peak, incl, w, h)
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-6)


def test_trace_geodesics_matches_oracle_paths(cuda, leg, oracle):
    from blackhole_b200._abi import default_scene

    a, r_obs, incl, steps, h = 0.9, 60.0, 1.2, 400, 0.5
    xyz, cnt = leg.trace_geodesics(a, r_obs, incl, (-8.0, 8.0, 5), (-6.0, 6.0, 4), steps, h)
    s = default_scene(width=5, height=4, spin=a, theta_obs=incl, integrator=0, max_crossings=1, precision=0)
    s.r_obs = r_obs
    s.potential_form = 1
    s.step_coeff = h / 20.0
    s.step_rcap = 20.0
    i, j = np.meshgrid(np.arange(5), np.arange(4))
    alpha = (-8.0 + 16.0 * i / 4).ravel()
    beta = (-6.0 + 12.0 * j / 3).ravel()
    rxyz, rcnt = oracle.trace_paths(s, alpha, beta, steps)
    np.testing.assert_array_equal(cnt, rcnt)
    assert cnt.min() >= 2
    for k in range(len(cnt)):
        np.testing.assert_allclose(xyz[k, :cnt[k]], rxyz[k, :cnt[k]], rtol=1e-5, atol=1e-4)
