"""The reference renderer's launch ABI on the GPU (include/bh_legacy.h), through
the C ABI: camera rays, shading, the backend, the Blender-bridge calls, the
post-processing, the lensing map, the disk texture and the geodesic paths,
each against the CPU oracle (kerr_oracle.hpp camera/paths,
oracle/legacy_oracle.py shading and post-processing), and the post-processing
also against the reference's own kernels (oracle/_ref/libbh_ref_post.so, built
from src/blender_bridge/cuda_postprocess.cu), and the disk geometry of the
render against the reference's own render kernels
(oracle/_ref/libbh_ref_render.so, built from src/cuda)."""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import legacy_oracle as LO

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def leg():
    """The bindings, with the physical shading these tests pin (the reference
    look, the default, is pinned in test_gpu_legacy_look.py)."""
    from blackhole_b200 import legacy

    legacy.library()
    before = legacy.get_shading()
    legacy.set_shading(legacy.SHADING_PHYSICAL)
    yield legacy
    legacy.set_shading(before)


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


def _gather_source(w: int, h: int) -> np.ndarray:
    """Flat index of the pixel each pixel's red and blue come from in the tone map."""
    f32 = np.float32
    rx = np.floor((np.arange(w, dtype=f32) / f32(w)) * f32(w)).astype(np.int64)
    ry = np.floor((np.arange(h, dtype=f32) / f32(h)) * f32(h)).astype(np.int64)
    return (ry[:, None] * w + rx[None, :]).ravel()


def test_bridge_render_is_postprocessed_shading(cuda, leg, oracle, monkeypatch):
    for var in ("BLACKHOLE_BRIDGE_EXPOSURE", "BLACKHOLE_BRIDGE_BLOOM_STRENGTH", "BLACKHOLE_BRIDGE_BLOOM_THRESHOLD"):
        monkeypatch.delenv(var, raising=False)
    spin, r_rs, incl, w, h = 0.8, 25.0, 1.25, 47, 36  # width 47: six columns take red and blue from the left
    img = leg.render_raytraced(spin, r_rs, incl, w, h).reshape(-1, 4)
    p = leg.bridge_params(spin, r_rs, incl, 1.0, w, h)
    ref, cf = _oracle_frame(oracle, p)
    want = LO.postprocess(LO.shade(ref, p, cf[15], cf[16]).reshape(h, w, 4), 1.0, 0.0, 12.0).reshape(-1, 4)
    assert np.all(img[:, 3] == 1.0) and img.min() >= 0.0 and img.max() <= 1.0
    src = _gather_source(w, h)
    assert (src != np.arange(w * h)).any()
    agree = (img[:, 1] > 0) == (ref["cls"] == 1)  # green is the pixel's own
    assert agree.mean() >= 0.99
    ok = agree & agree[src]
    np.testing.assert_allclose(img[ok], want[ok], rtol=2e-4, atol=2e-6)
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


def _hdr_frame(w: int, h: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    fb = rng.lognormal(-1.0, 1.5, (h, w, 4)).astype(np.float32)
    fb[rng.random((h, w)) < 0.3] = 0.0  # black patches: luminance below 0.001
    fb[..., 3] = rng.random((h, w)).astype(np.float32)
    return fb


@pytest.mark.parametrize("w,h,threshold,strength,exposure", [
    (61, 37, 0.8, 0.6, 3.0), (130, 96, 1.0, 0.0, 12.0), (200, 70, 0.25, 1.5, 0.7), (5, 3, 0.5, 1.0, 2.0),
    (1, 1, 0.1, 2.0, 1.0), (64, 200, 1.0, 0.3, 12.0)])
def test_postprocess_matches_restatement(cuda, leg, w, h, threshold, strength, exposure):
    fb = _hdr_frame(w, h, w * 1000 + h)
    d = torch.from_numpy(fb).cuda().reshape(-1)
    leg.postprocess(d, w, h, threshold, strength, exposure, 0.5)
    got = d.cpu().numpy().reshape(h, w, 4)
    want = LO.postprocess(fb, threshold, strength, exposure)
    np.testing.assert_allclose(got, want, rtol=2e-5, atol=1e-6)


def test_postprocess_rejects_bad_arguments(cuda, leg):
    L = leg.library()
    assert L.bhb_cuda_postprocess(None, 4, 4, 1.0, 0.0, 1.0, 0.0) == -1
    d = torch.zeros(16 * 4, device="cuda")
    assert L.bhb_cuda_postprocess(C.c_void_p(d.data_ptr()), 0, 4, 1.0, 0.0, 1.0, 0.0) == -1
    assert L.bhb_cuda_postprocess(C.c_void_p(d.data_ptr()), 4, -1, 1.0, 0.0, 1.0, 0.0) == -1


REF_POST = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libbh_ref_post.so"


@pytest.mark.skipif(not REF_POST.exists(), reason="reference post-processing build absent (oracle/_ref)")
@pytest.mark.parametrize("w,h,threshold,strength,exposure", [(61, 37, 0.8, 0.6, 3.0), (160, 90, 1.0, 0.0, 12.0),
                                                             (96, 130, 0.3, 1.2, 1.5)])
def test_postprocess_matches_reference_build(cuda, leg, w, h, threshold, strength, exposure):
    """Against the reference's own bhb_cuda_postprocess, compiled from its
    source. Its tone map reads the left or upper neighbour's red and blue in
    place, racing with that neighbour's write; those pixels are excluded."""
    ref_lib = C.CDLL(str(REF_POST))
    ref_lib.bhb_cuda_postprocess.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                             C.c_float]
    fb = _hdr_frame(w, h, 7 * w + h)
    a = torch.from_numpy(fb).cuda().reshape(-1)
    b = a.clone()
    torch.cuda.synchronize()
    assert ref_lib.bhb_cuda_postprocess(C.c_void_p(a.data_ptr()), w, h, threshold, strength, exposure, 0.0) == 0
    torch.cuda.synchronize()
    leg.postprocess(b, w, h, threshold, strength, exposure, 0.0)
    ra, rb = a.cpu().numpy().reshape(-1, 4), b.cpu().numpy().reshape(-1, 4)
    own = _gather_source(w, h) == np.arange(w * h)
    assert own.mean() > 0.75
    np.testing.assert_allclose(rb[own], ra[own], rtol=2e-5, atol=1e-6)
    np.testing.assert_allclose(rb[:, 1], ra[:, 1], rtol=2e-5, atol=1e-6)  # green is always the pixel's own


REF_RENDER = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libbh_ref_render.so"


def _grow(m, k):
    out = m.copy()
    for dy in range(-k, k + 1):
        for dx in range(-k, k + 1):
            out |= np.roll(np.roll(m, dy, 0), dx, 1)
    return out


@pytest.mark.skipif(not REF_RENDER.exists(), reason="reference render-kernel build absent (oracle/_ref)")
@pytest.mark.parametrize("spin,r_rs,incl", [(0.0, 15.0, 1.3), (0.0, 10.0, 1.5), (0.9, 15.0, 1.3), (0.5, 12.0, 1.45)])
def test_disk_geometry_against_reference_render_kernel(cuda, leg, spin, r_rs, incl):
    """Which pixels see the disk, ours against the reference's own FP32 kernel
    (geodesicTraceFp32, src/cuda/kernels_fp32.cu:35, through its
    bh_launch_geodesic_kernel, compiled from its source) on the same
    BH_LaunchParams: Kerr stepping on, background and photon glow off, so that
    both paint exactly the disk pixels (device_physics.cuh:1522-1525 black
    background, :1899-1924 glow scaled by photon_glow_strength; disk z = 0
    between isco and 30 rs, :606-613 and :936-937).

    a = 0: the images agree except within 3 pixels of the disk's edges (the
    reference's FP32 steps cross the plane with a coarse linear interpolation
    at the outer rim). a != 0: the reference paints no disk below the shadow
    (the near side of the disk, seen through the first plane crossing), while
    the far side above it agrees; nothing it paints is absent from ours."""
    ref_lib = C.CDLL(str(REF_RENDER))
    ref_lib.bh_launch_geodesic_kernel.argtypes = [C.c_void_p, C.POINTER(leg.LaunchParams), C.c_int, C.c_void_p]
    ref_lib.bh_launch_geodesic_kernel.restype = C.c_int
    p = leg.bridge_params(spin, r_rs, incl, 0.6, 160, 120)
    p.kerr_enabled = 1
    p.background_enabled = 0
    p.photon_glow_strength = 0.0
    p.max_steps = 20000
    p.step_size = 0.04
    fb = torch.zeros(p.height * p.width * 4, dtype=torch.float32, device="cuda")
    assert ref_lib.bh_launch_geodesic_kernel(C.c_void_p(fb.data_ptr()), C.byref(p), 0, None) == 0
    torch.cuda.synchronize()
    theirs = fb.view(p.height, p.width, 4).cpu().numpy()
    ours = _render(leg, p).reshape(p.height, p.width, 4)
    assert np.all(np.isfinite(theirs)) and np.all(np.isfinite(ours))
    d_ours, d_ref = ours[..., :3].sum(-1) > 0, theirs[..., :3].sum(-1) > 0
    diff = d_ours != d_ref
    half = p.height // 2
    if spin == 0.0:
        assert d_ours.mean() > 0.5 and np.mean(~diff) >= 0.95, np.mean(~diff)
        assert not np.any(diff & ~(_grow(d_ours, 3) & _grow(~d_ours, 3)))
    else:
        assert np.mean(~diff[:half]) >= 0.995, np.mean(~diff[:half])
        assert d_ours[half:].mean() > 0.3 and not d_ref[half:].any()
        assert np.mean(d_ref & ~d_ours) < 1e-3


def test_bridge_environment_overrides(cuda, leg, oracle, monkeypatch):
    """BLACKHOLE_BRIDGE_* variables reach the render and the post-processing
    (src/blender_bridge/cuda_renderer.cu:425-552, 665-673): exposure 3 and
    disk brightness 0.7 give the oracle's frame with those settings; an
    unparsable value keeps the default."""
    spin, r_rs, incl, w, h = 0.6, 30.0, 1.1, 40, 30
    monkeypatch.setenv("BLACKHOLE_BRIDGE_EXPOSURE", "3")
    monkeypatch.setenv("BLACKHOLE_BRIDGE_ADISK_LIT", "0.7")
    monkeypatch.setenv("BLACKHOLE_BRIDGE_BLOOM_STRENGTH", "not-a-number")
    img = leg.render_raytraced(spin, r_rs, incl, w, h).reshape(-1, 4)
    p = leg.bridge_params(spin, r_rs, incl, 1.0, w, h)
    p.adisk_lit = 0.7
    ref, cf = _oracle_frame(oracle, p)
    want = LO.postprocess(LO.shade(ref, p, cf[15], cf[16]).reshape(h, w, 4), 1.0, 0.0, 3.0).reshape(-1, 4)
    agree = (img[:, 1] > 0) == (ref["cls"] == 1)
    assert agree.mean() >= 0.99
    ok = agree & agree[_gather_source(w, h)]
    np.testing.assert_allclose(img[ok], want[ok], rtol=2e-4, atol=2e-6)
    monkeypatch.setenv("BLACKHOLE_BRIDGE_ADISK_ENABLED", "off")
    dark = leg.render_raytraced(spin, r_rs, incl, w, h).reshape(-1, 4)
    assert np.all(dark[:, :3] == 0.0)  # no disk, no background texture: black
