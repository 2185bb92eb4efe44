"""Python host API of the B200 Kerr tracer (a thin layer over include/bh_kerr.h).

Two groups, mirroring the reference:

* ``KerrRaytracer``, ``kerr_potentials``, ``kerr_step_mino`` - batched GPU
  versions of physics::KerrRaytracer / kerrPotentials / kerrStepMino
  (src/physics/raytracer.h:309-399, src/physics/kerr.cpp:40-134), CGS units,
  taking torch CUDA tensors (structure of arrays).
* ``trace_image`` / ``trace_image_host`` - the image-plane tracer in
  geometric units (M = 1).

All compute runs in the CUDA library; nothing here falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _abi
from ._abi import KerrConstsSoA, KerrImageOut, KerrRaytracerParams, KerrScene, KerrStateSoA, check

STATE_FIELDS = ("r", "theta", "phi", "t", "sign_r", "sign_theta")


def _stream_ptr(stream) -> int | None:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


def _f64(t: torch.Tensor, name: str) -> torch.Tensor:
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous():
        raise TypeError(f"{name} must be a contiguous float64 CUDA tensor")
    return t


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def scene(**overrides) -> KerrScene:
    """A BH_KerrScene filled with the library defaults, then ``overrides``."""
    s = KerrScene()
    _abi.load_library().bh_kerr_scene_defaults(C.byref(s))
    for k, v in overrides.items():
        if not hasattr(s, k):
            raise AttributeError(f"BH_KerrScene has no field {k!r}")
        setattr(s, k, v)
    return s


def validate(s: KerrScene) -> None:
    check(_abi.load_library().bh_kerr_scene_validate(C.byref(s)))


def alloc_image_outputs(s: KerrScene, device="cuda", fields=None) -> dict[str, torch.Tensor]:
    """Device output tensors for a scene (all fields unless ``fields`` is given)."""
    n = s.width * s.height
    mc = s.max_crossings
    shapes = {
        "cls": ((n,), torch.int32), "steps": ((n,), torch.int32), "n_cross": ((n,), torch.int32),
        "r_hit": ((mc, n), torch.float64), "phi_hit": ((mc, n), torch.float64), "g": ((mc, n), torch.float64),
        "flux": ((n,), torch.float64), "intensity": ((n,), torch.float64),
        "theta_inf": ((n,), torch.float64), "phi_inf": ((n,), torch.float64),
        "carter_drift": ((n,), torch.float64),
    }
    fields = fields or list(_abi.OUT_FIELDS)
    return {k: torch.empty(*shapes[k][0], dtype=shapes[k][1], device=device) for k in fields}


def _out_struct(outs: dict) -> KerrImageOut:
    o = KerrImageOut()
    for k, v in outs.items():
        setattr(o, k, v.data_ptr() if isinstance(v, torch.Tensor) else v.ctypes.data)
    return o


def sky_generate(size: int = 512, n_stars: int = 10_000, seed: int = 1, device="cuda", stream=None) -> torch.Tensor:
    """The seeded background sky (bh_sky_generate): FP16 cubemap [6][size][size]."""
    tex = torch.empty(6, size, size, dtype=torch.float16, device=device)
    check(_abi.load_library().bh_sky_generate(tex.data_ptr(), size, n_stars, seed, _stream_ptr(stream)))
    return tex


def _sky_struct(sky: torch.Tensor | None):
    if sky is None:
        return None
    if sky.dtype != torch.float16 or not sky.is_cuda or sky.dim() != 3 or sky.shape[0] != 6:
        raise TypeError("sky must be a CUDA float16 tensor [6][N][N]")
    return _abi.SkyCubemap(sky.data_ptr(), sky.shape[1], 0)


def trace_image(s: KerrScene, outs: dict[str, torch.Tensor] | None = None, stream=None,
                sky: torch.Tensor | None = None) -> dict[str, torch.Tensor]:
    """Trace every pixel of ``s`` on the current CUDA device (asynchronous).

    ``outs`` maps BH_KerrImageOut field names to device tensors; missing
    fields are not written. Allocates all fields when ``outs`` is None.
    ``sky``: a cubemap (sky_generate) whose radiance escaped rays add to
    their intensity.
    """
    if outs is None:
        outs = alloc_image_outputs(s)
    for k, v in outs.items():
        if k not in _abi.DEVICE_OUT_FIELDS:
            raise KeyError(f"unknown output field {k!r}")
        if not v.is_cuda or not v.is_contiguous():
            raise TypeError(f"output {k} must be a contiguous CUDA tensor")
    o = _out_struct(outs)
    if sky is not None:
        check(_abi.load_library().bh_kerr_trace_image_sky(C.byref(s), C.byref(o), C.byref(_sky_struct(sky)),
                                                          _stream_ptr(stream)))
    else:
        check(_abi.load_library().bh_kerr_trace_image(C.byref(s), C.byref(o), _stream_ptr(stream)))
    return outs


def host_image_outputs(s: KerrScene, fields=None):
    """Zeroed host (numpy) output arrays of a scene and their BH_KerrImageOut."""
    n = s.width * s.height
    mc = s.max_crossings
    dt = {"cls": np.int32, "steps": np.int32, "n_cross": np.int32}
    fields = fields or _abi.OUT_FIELDS
    outs = {}
    for k in fields:
        shape = (mc, n) if k in _abi.PLANE_FIELDS else (n,)
        outs[k] = np.zeros(shape, dt.get(k, np.float64))
    return outs, _out_struct(outs)


def trace_image_host(s: KerrScene, fields=None) -> dict[str, np.ndarray]:
    """Trace into host (numpy) arrays through bh_kerr_trace_image_host."""
    outs, o = host_image_outputs(s, fields)
    check(_abi.load_library().bh_kerr_trace_image_host(C.byref(s), C.byref(o)))
    return outs


def trace_image_host_noalloc(s: KerrScene, fields=None, stream=None) -> dict[str, np.ndarray]:
    """Trace into host arrays through bh_kerr_trace_image_host_noalloc.

    Allocates no device memory: the outputs are staged in the library's fixed
    32 MiB device scratch, so images whose outputs exceed it are rejected.
    ``stream``: a torch.cuda.Stream, a raw cudaStream_t, or None for the
    legacy default stream.
    """
    n = s.width * s.height
    mc = s.max_crossings
    dt = {"cls": np.int32, "steps": np.int32, "n_cross": np.int32}
    fields = fields or _abi.OUT_FIELDS
    outs = {}
    for k in fields:
        shape = (mc, n) if k in _abi.PLANE_FIELDS else (n,)
        outs[k] = np.zeros(shape, dt.get(k, np.float64))
    sp = None if stream is None else (stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
    check(_abi.load_library().bh_kerr_trace_image_host_noalloc(C.byref(s), C.byref(_out_struct(outs)), sp))
    return outs


def set_launch(block_threads: int = 0, ctas_per_sm: int = 0) -> None:
    """Override the persistent-grid shape (0 = automatic)."""
    check(_abi.load_library().bh_kerr_set_launch(block_threads, ctas_per_sm))


class TraceBatch:
    """Many frames of uneven size traced by one persistent launch
    (BH_KerrBatch). All scenes share integrator and precision.

    ``outs``: one dict of device tensors per frame (allocated when None).
    """

    def __init__(self, scenes, outs=None, device="cuda", fields=None):
        self.scenes = list(scenes)
        if not self.scenes:
            raise ValueError("a batch needs at least one frame")
        self.outs = outs if outs is not None else [alloc_image_outputs(s, device=device, fields=fields)
                                                   for s in self.scenes]
        n = len(self.scenes)
        sarr = (KerrScene * n)(*self.scenes)
        oarr = (KerrImageOut * n)(*[_out_struct(o) for o in self.outs])
        lib = _abi.load_library()
        h = lib.bh_kerr_batch_create(sarr, oarr, n)
        if not h:
            raise RuntimeError(lib.bh_last_error().decode())
        self._h = h
        self._lib = lib

    def __len__(self):
        return len(self.scenes)

    @property
    def pixels(self) -> int:
        return int(self._lib.bh_kerr_batch_pixels(self._h))

    def trace(self, stream=None):
        check(self._lib.bh_kerr_batch_trace(self._h, _stream_ptr(stream)))
        return self.outs

    def trace_graph(self, stream=None):
        """Trace through a captured CUDA graph (captured on first use)."""
        check(self._lib.bh_kerr_batch_trace_graph(self._h, _stream_ptr(stream)))
        return self.outs

    def set_sky(self, sky: torch.Tensor | None):
        """Attach a sky cubemap to every frame (None detaches)."""
        self._sky = sky  # keep the texels alive
        st = _sky_struct(sky)
        check(self._lib.bh_kerr_batch_set_sky(self._h, C.byref(st) if st is not None else None))

    def set_launch(self, block_threads=0, ctas_per_sm=0, refill_steps=1):
        cfg = _abi.KerrLaunchConfig(block_threads, ctas_per_sm, refill_steps, 0)
        check(self._lib.bh_kerr_batch_set_launch(self._h, C.byref(cfg)))

    def launch(self) -> dict:
        cfg = _abi.KerrLaunchConfig()
        check(self._lib.bh_kerr_batch_get_launch(self._h, C.byref(cfg)))
        return {"block_threads": cfg.block_threads, "ctas_per_sm": cfg.ctas_per_sm, "refill_steps": cfg.refill_steps}

    def autotune(self, max_pixels=0, stream=None) -> dict:
        cfg = _abi.KerrLaunchConfig()
        check(self._lib.bh_kerr_batch_autotune(self._h, max_pixels, _stream_ptr(stream), C.byref(cfg)))
        return {"block_threads": cfg.block_threads, "ctas_per_sm": cfg.ctas_per_sm, "refill_steps": cfg.refill_steps}

    def frame_times(self) -> np.ndarray:
        """Per-frame completion times (ms after the launch started) of the last trace."""
        out = np.zeros(len(self.scenes), np.float32)
        check(self._lib.bh_kerr_batch_frame_times(self._h, out.ctypes.data))
        return out

    def close(self):
        if getattr(self, "_h", None):
            self._lib.bh_kerr_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass


# --------------------------------------------------------------------------
# src/physics API, batched
# --------------------------------------------------------------------------

def _state_soa(state: dict) -> KerrStateSoA:
    s = KerrStateSoA()
    for k in STATE_FIELDS:
        setattr(s, k, _f64(state[k], k).data_ptr())
    return s


def _consts_soa(e, lz, q) -> KerrConstsSoA:
    c = KerrConstsSoA()
    c.e, c.lz, c.q = _f64(e, "e").data_ptr(), _f64(lz, "lz").data_ptr(), _f64(q, "q").data_ptr()
    return c


def kerr_potentials(r, theta, mass: float, a: float, e, lz, q, stream=None) -> dict[str, torch.Tensor]:
    """Batched physics::kerrPotentials (kerr.cpp:69-97): R, dR/dr, Theta, dTheta/dtheta."""
    n = _f64(r, "r").numel()
    _f64(theta, "theta")
    out = {k: torch.empty(n, dtype=torch.float64, device=r.device) for k in ("r_pot", "dr_pot", "theta_pot", "dtheta_pot")}
    check(_abi.load_library().bh_kerr_potentials(
        n, r.data_ptr(), theta.data_ptr(), mass, a, _consts_soa(e, lz, q),
        out["r_pot"].data_ptr(), out["dr_pot"].data_ptr(), out["theta_pot"].data_ptr(), out["dtheta_pot"].data_ptr(),
        _stream_ptr(stream)))
    return out


def kerr_step_mino(state: dict, mass: float, a: float, e, lz, q, dlam, stream=None) -> dict:
    """Batched physics::kerrStepMino (kerr.cpp:99-134), in place on ``state``."""
    n = state["r"].numel()
    if isinstance(dlam, torch.Tensor):
        dptr, dscalar = _f64(dlam, "dlam").data_ptr(), 0.0
    else:
        dptr, dscalar = None, float(dlam)
    check(_abi.load_library().bh_kerr_step_mino(n, _state_soa(state), mass, a, _consts_soa(e, lz, q), dptr, dscalar,
                                                 _stream_ptr(stream)))
    return state


@dataclass
class RayTraceResult:
    """Batched physics::RayTraceResult (raytracer.h:72-79), one entry per ray."""

    status: torch.Tensor
    steps_taken: torch.Tensor
    total_distance: torch.Tensor
    final_r: torch.Tensor
    final_theta: torch.Tensor
    final_phi: torch.Tensor
    redshift: torch.Tensor


class KerrRaytracer:
    """physics::KerrRaytracer (src/physics/raytracer.h:309-399), batched on the GPU.

    Same constructor defaults (horizon, escape radius 1000 r_s, step 0.02 r_s,
    10000 steps) and setters; ``trace`` takes a batch of states and constants.
    """

    def __init__(self, mass: float, spin_param: float):
        self._p = KerrRaytracerParams()
        check(_abi.load_library().bh_kerr_raytracer_defaults(mass, spin_param, C.byref(self._p)))

    def set_step_size(self, h: float) -> None:
        self._p.step_size = h

    def set_max_steps(self, n: int) -> None:
        self._p.max_steps = n

    def set_escape_radius(self, r: float) -> None:
        self._p.r_escape = r

    @property
    def params(self) -> KerrRaytracerParams:
        return self._p

    def trace(self, initial: dict, e, lz, q, stream=None) -> RayTraceResult:
        n = initial["r"].numel()
        dev = initial["r"].device
        st = torch.empty(n, dtype=torch.int32, device=dev)
        steps = torch.empty(n, dtype=torch.int32, device=dev)
        f = [torch.empty(n, dtype=torch.float64, device=dev) for _ in range(5)]
        check(_abi.load_library().bh_kerr_trace_rays(
            n, _state_soa(initial), _consts_soa(e, lz, q), C.byref(self._p),
            st.data_ptr(), steps.data_ptr(), *[x.data_ptr() for x in f], _stream_ptr(stream)))
        return RayTraceResult(st, steps, f[0], f[1], f[2], f[3], f[4])
