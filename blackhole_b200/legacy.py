"""The reference renderer's launch ABI (include/bh_legacy.h) from Python.

A ctypes mirror of ``BH_LaunchParams`` (the byte layout of the reference's
src/cuda/kernel_launch.h), the Blender bridge's camera orbit, and thin
wrappers over ``bh_launch_geodesic_kernel`` and the ``bhbCuda*`` calls, in the
style of the reference add-on's ctypes binding
(blender/addon/blackhole_physics/render_engine.py:42-68).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._abi import check, load_library

_f, _i = C.c_float, C.c_int


class LaunchParams(C.Structure):
    _fields_ = [
        ("rs", _f), ("spin", _f), ("isco", _f), ("step_size", _f), ("fov_scale", _f), ("max_dist", _f),
        ("cam_pos", _f * 3), ("cam_basis", _f * 9), ("frame_shift_x", _f), ("frame_shift_y", _f),
        ("max_steps", _i), ("width", _i), ("height", _i),
        ("adisk_enabled", _i), ("redshift_enabled", _i), ("kerr_enabled", _i), ("use_luts", _i),
        ("lut_radius_min", _f), ("lut_radius_max", _f), ("redshift_radius_min", _f), ("redshift_radius_max", _f),
        ("spectral_radius_min", _f), ("spectral_radius_max", _f),
        ("time_sec", _f), ("doppler_strength", _f), ("background_intensity", _f), ("background_enabled", _i),
        ("photon_glow_strength", _f),
        ("debug_pre_redshift_background", _i), ("debug_pre_shaping_background", _i),
        ("debug_post_shaping_background", _i), ("debug_shaper_inputs", _i), ("debug_closest_approach_state", _i),
        ("debug_closest_approach_timeline", _i), ("debug_closest_approach_direction", _i),
        ("debug_escaped_direction", _i),
        ("background_yaw_rad", _f), ("background_pitch_rad", _f), ("background_filter_radius", _f),
        ("background_layer_params", _f * 12), ("background_layer_lod_bias", _f * 3),
        ("wiregrid_enabled", _i), ("wiregrid_show_ergo", _f), ("wiregrid_grid_scale", _f),
        ("wiregrid_motion_scale", _f), ("wiregrid_infall_scale", _f), ("wiregrid_strength", _f),
        ("wiregrid_scene_preserve", _f), ("wiregrid_color", _f * 4),
        ("grmhd_r_min", _f), ("grmhd_r_max", _f), ("rte_enabled", _i), ("rte_opacity_scale", _f),
        ("grmhd_alpha", _f), ("stokes_enabled", _i), ("stokes_b_field_angle", _f), ("stokes_ne_scale", _f),
        ("adisk_lit", _f),
    ]


class DiskParams(C.Structure):
    _fields_ = [("aStar", C.c_double), ("massMsun", C.c_double), ("mdotEdd", C.c_double), ("rOutRg", C.c_double),
                ("inclinationRad", C.c_double)]


def isco_prograde(a: float) -> float:
    """Bardeen-Press-Teukolsky prograde ISCO [M]."""
    z1 = 1 + (1 - a * a) ** (1 / 3) * ((1 + a) ** (1 / 3) + (1 - a) ** (1 / 3))
    z2 = math.sqrt(3 * a * a + z1 * z1)
    return 3 + z2 - math.sqrt((3 - z1) * (3 + z1 + 2 * z2))


def bridge_isco_rs(spin: float) -> float:
    """The bridge's ISCO in rs, in float32 (src/blender_bridge/cuda_renderer.cu:433-439)."""
    f32 = np.float32
    a = f32(spin)
    third = f32(1.0) / f32(3.0)
    z1 = f32(1) + np.power(f32(1) - a * a, third) * (np.power(f32(1) + a, third) + np.power(f32(1) - a, third))
    z2 = np.sqrt(f32(3) * a * a + z1 * z1)
    return float(f32(0.5) * (f32(3) + z2 - np.sqrt((f32(3) - z1) * (f32(3) + z1 + f32(2) * z2))))


def bridge_params(spin: float, observer_r: float, incl: float, fov: float, width: int, height: int) -> LaunchParams:
    """The Blender bridge's camera and defaults with no BLACKHOLE_BRIDGE_*
    overrides set (legacy_api.cpp bridge_params, after
    src/blender_bridge/cuda_renderer.cu:425-552): camera on the (y, z) circle
    of radius observer_r [rs] at the inclination from +z, looking at the
    origin, basis columns right = forward x (0, 1, 0), up, forward."""
    f32 = np.float32
    p = LaunchParams()
    p.rs = 1.0
    p.spin = spin
    p.isco = bridge_isco_rs(spin)
    p.step_size = 0.08
    p.fov_scale = max(fov, 0.05)
    p.max_dist = 500.0
    p.max_steps = 600
    p.width, p.height = width, height
    ci, si = f32(math.cos(incl)), f32(math.sin(incl))
    p.cam_pos[:] = [0.0, f32(observer_r) * si, f32(observer_r) * ci]
    fw = np.array([0.0, -si, -ci], f32)
    r = np.array([-fw[2], 0.0, fw[0]], f32)
    rl = np.sqrt(np.sum(r * r, dtype=f32))
    if rl < 1e-6:
        r, rl = np.array([1.0, 0.0, 0.0], f32), f32(1.0)
    r = r / rl
    u = np.array([r[1] * fw[2] - r[2] * fw[1], r[2] * fw[0] - r[0] * fw[2], r[0] * fw[1] - r[1] * fw[0]], f32)
    p.cam_basis[:] = [float(v) for v in np.concatenate([r, u, fw])]
    p.adisk_enabled = 1
    p.redshift_enabled = 1
    p.kerr_enabled = 1 if abs(spin) > 1e-6 else 0
    p.doppler_strength = 1.0
    p.background_intensity = 0.8
    p.background_enabled = 1
    p.photon_glow_strength = 1.0
    drift, parallax = f32(0.01), f32(0.0006)
    for i, (depth, scale, inten, lod) in enumerate(((0.2, 1.0, 1.0, 0.0), (0.5, 1.08, 0.6, 1.0),
                                                    (0.9, 1.16, 0.35, 2.0))):
        p.background_layer_params[4 * i:4 * i + 4] = [
            float(drift + f32(p.cam_pos[0]) * parallax * f32(depth)),
            float(f32(0.0) + f32(p.cam_pos[1]) * parallax * f32(depth)), scale, inten]
        p.background_layer_lod_bias[i] = lod
    p.adisk_lit = 0.35
    return p


def _declare(lib: C.CDLL) -> C.CDLL:
    if getattr(lib, "_legacy_declared", False):
        return lib
    vp, f, d, i = C.c_void_p, C.c_float, C.c_double, C.c_int
    lib.bh_launch_geodesic_kernel.argtypes = [vp, C.POINTER(LaunchParams), i, vp]
    lib.bh_upload_lut_textures.argtypes = [C.c_ulonglong] * 8
    lib.bh_upload_lut_textures.restype = None
    lib.bh_upload_bridge_background_texture.argtypes = [C.c_ulonglong]
    lib.bh_upload_bridge_background_texture.restype = None
    lib.bhCudaInit.restype = vp
    lib.bhCudaInit.argtypes = [C.c_uint, i, i]
    lib.bhCudaRenderFrame.argtypes = [vp, C.POINTER(LaunchParams)]
    lib.bhCudaResize.argtypes = [vp, C.c_uint, i, i]
    lib.bhCudaRegisterLut.argtypes = [vp, i, C.c_uint, C.c_uint]
    lib.bhCudaRegisterBackgroundTexture.argtypes = [vp, C.c_uint, C.c_uint]
    lib.bhCudaSetVariant.argtypes = [vp, i]
    lib.bhCudaGetVariant.argtypes = [vp]
    lib.bhCudaShutdown.argtypes = [vp]
    lib.bhCudaShutdown.restype = None
    lib.bhCudaFramebuffer.argtypes = [vp]
    lib.bhCudaFramebuffer.restype = vp
    lib.bhbCudaRenderRaytraced.argtypes = [f, f, f, i, i, vp]
    lib.bhbCudaRenderRaytracedCamera.argtypes = [f, f, f, f, i, i, vp]
    lib.bhbCudaRenderRaytracedView.argtypes = [f, vp, vp, f, i, i, vp]
    lib.bhbCudaRenderLensingMap.argtypes = [d, d, d, i, i, vp]
    lib.bhbCudaRenderDiskTexture.argtypes = [C.POINTER(DiskParams), i, i, vp]
    lib.bhbCudaTraceGeodesics.argtypes = [d, d, d, d, d, i, d, d, i, i, d, vp, vp]
    for name in ("bhb_cuda_render_raytraced", "bhb_cuda_render_raytraced_camera"):
        getattr(lib, name).argtypes = lib.bhbCudaRenderRaytraced.argtypes if "camera" not in name else \
            lib.bhbCudaRenderRaytracedCamera.argtypes
    lib.bhb_cuda_render_raytraced_view.argtypes = lib.bhbCudaRenderRaytracedView.argtypes
    lib.bhb_cuda_render_lensing_map.argtypes = [f, f, f, i, i, vp]
    lib.bhb_cuda_render_disk_texture.argtypes = [f, f, f, i, i, vp]
    lib.bhb_cuda_postprocess.argtypes = [vp, i, i, f, f, f, f]
    lib.bh_legacy_set_shading.argtypes = [i]
    lib.bh_legacy_get_shading.argtypes = []
    lib.bh_stokes_steps.argtypes = [C.c_int64, vp, vp, vp, vp]
    lib._legacy_declared = True
    return lib


def library() -> C.CDLL:
    return _declare(load_library())


SHADING_REFERENCE, SHADING_PHYSICAL = 0, 1


def set_shading(mode: int) -> None:
    """Colour of the render calls: SHADING_REFERENCE (the reference shader's
    look, the default) or SHADING_PHYSICAL (bh_legacy_set_shading)."""
    check(library().bh_legacy_set_shading(int(mode)))


def get_shading() -> int:
    return int(library().bh_legacy_get_shading())


def stokes_steps(state, coef, stream=None):
    """bh_stokes_steps: one exact polarized transfer step for each row of
    ``state`` [n, 4] (I, Q, U, V) with ``coef`` [n, 7] (jI, jQ, jU, jV,
    alpha_I, rho_V, ds); contiguous float32 CUDA tensors. Returns [n, 4]."""
    import torch

    if state.dtype != torch.float32 or coef.dtype != torch.float32 or not state.is_cuda or not coef.is_cuda:
        raise TypeError("state and coef must be float32 CUDA tensors")
    if state.dim() != 2 or state.shape[1] != 4 or coef.shape != (state.shape[0], 7):
        raise ValueError("state must be [n, 4] and coef [n, 7]")
    state, coef = state.contiguous(), coef.contiguous()
    out = torch.empty_like(state)
    s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    check(library().bh_stokes_steps(state.shape[0], state.data_ptr(), coef.data_ptr(), out.data_ptr(), s))
    return out


def launch(params: LaunchParams, framebuffer, variant: int = -1, stream=None) -> None:
    """bh_launch_geodesic_kernel into a device float4 buffer (a torch tensor
    of width * height * 4 float32 on the current device)."""
    lib = library()
    s = None if stream is None else C.c_void_p(stream.cuda_stream)
    check(lib.bh_launch_geodesic_kernel(C.c_void_p(framebuffer.data_ptr()), C.byref(params), variant, s))


def render_raytraced(spin: float, observer_r: float, incl: float, width: int, height: int,
                     fov: float | None = None) -> np.ndarray:
    """bhbCudaRenderRaytraced(Camera): host RGBA [height, width, 4]."""
    lib = library()
    out = np.zeros((height, width, 4), np.float32)
    if fov is None:
        check(lib.bhbCudaRenderRaytraced(spin, observer_r, incl, width, height, out.ctypes.data))
    else:
        check(lib.bhbCudaRenderRaytracedCamera(spin, observer_r, incl, fov, width, height, out.ctypes.data))
    return out


def postprocess(framebuffer, width: int, height: int, bloom_threshold: float = 1.0, bloom_strength: float = 0.0,
                exposure_gain: float = 12.0, time_sec: float = 0.0) -> None:
    """bhb_cuda_postprocess in place on a device float4 framebuffer (a torch
    tensor of width * height * 4 float32 on the current device)."""
    lib = library()
    check(lib.bhb_cuda_postprocess(C.c_void_p(framebuffer.data_ptr()), width, height, bloom_threshold,
                                   bloom_strength, exposure_gain, time_sec))


def lensing_map(a: float, r_obs: float, incl: float, width: int, height: int) -> np.ndarray:
    lib = library()
    out = np.zeros((height, width, 4), np.float32)
    check(lib.bhbCudaRenderLensingMap(a, r_obs, incl, width, height, out.ctypes.data))
    return out


def disk_texture(a: float, r_out: float, incl: float, width: int, height: int) -> np.ndarray:
    lib = library()
    out = np.zeros((height, width, 4), np.float32)
    p = DiskParams(a, 1.0, 0.1, r_out, incl)
    check(lib.bhbCudaRenderDiskTexture(C.byref(p), width, height, out.ctypes.data))
    return out


def trace_geodesics(a: float, r_obs: float, incl: float, alpha: tuple[float, float, int],
                    beta: tuple[float, float, int], max_steps: int, step: float) -> tuple[np.ndarray, np.ndarray]:
    """bhbCudaTraceGeodesics: paths [n_beta * n_alpha, max_steps, 3] and point counts."""
    lib = library()
    n = alpha[2] * beta[2]
    xyz = np.zeros((n, max_steps, 3), np.float32)
    cnt = np.zeros(n, np.int32)
    check(lib.bhbCudaTraceGeodesics(a, r_obs, incl, alpha[0], alpha[1], alpha[2], beta[0], beta[1], beta[2],
                                    max_steps, step, xyz.ctypes.data, cnt.ctypes.data))
    return xyz, cnt
