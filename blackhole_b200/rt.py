"""Along-ray radiative transfer through a volumetric emitter (include/bh_rt.h).

The synthetic GRMHD-like medium (torus x exp of a Gaussian random field),
the thermal-synchrotron table and the traced image of I_nu. Tensors are
torch CUDA tensors (plumbing only).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _abi
from ._abi import KerrScene, check


class GrmhdGrid(C.Structure):
    _fields_ = [("cells", C.c_void_p), ("n_r", C.c_int32), ("n_theta", C.c_int32), ("n_phi", C.c_int32),
                ("reserved", C.c_int32), ("r_min", C.c_double), ("r_max", C.c_double)]


class TorusParams(C.Structure):
    _fields_ = [("r_in", C.c_double), ("r_peak", C.c_double), ("width", C.c_double), ("n0", C.c_double),
                ("theta0", C.c_double), ("b0", C.c_double), ("sigma", C.c_double), ("corr_len", C.c_double),
                ("seed", C.c_uint64)]


class SynchrotronLut(C.Structure):
    _fields_ = [("table", C.c_void_p), ("n_theta", C.c_int32), ("n_x", C.c_int32),
                ("log_theta_min", C.c_double), ("log_theta_max", C.c_double),
                ("log_x_min", C.c_double), ("log_x_max", C.c_double)]


class PackedGrmhdInfo(C.Structure):
    _fields_ = [("n_r", C.c_int32), ("n_theta", C.c_int32), ("n_phi", C.c_int32), ("reserved", C.c_int32),
                ("r_min", C.c_float), ("r_max", C.c_float), ("min_value", C.c_float * 4),
                ("max_value", C.c_float * 4), ("channels", (C.c_char * 32) * 4)]


class PackedConversion(C.Structure):
    _fields_ = [("n_scale", C.c_double), ("theta_scale", C.c_double), ("b_scale", C.c_double)]


class RtParams(C.Structure):
    _fields_ = [("nu_hz", C.c_double), ("length_cm", C.c_double), ("ds_max", C.c_double),
                ("min_transmit", C.c_double)]


def _lib():
    lib = _abi.load_library()
    if not getattr(lib, "_rt_declared", False):
        vp = C.c_void_p
        lib.bh_torus_defaults.restype = None
        lib.bh_torus_defaults.argtypes = [C.POINTER(TorusParams)]
        lib.bh_rt_defaults.restype = None
        lib.bh_rt_defaults.argtypes = [C.POINTER(RtParams)]
        lib.bh_grmhd_synthetic.restype = C.c_int
        lib.bh_grmhd_synthetic.argtypes = [C.POINTER(GrmhdGrid), C.POINTER(TorusParams), vp]
        lib.bh_synchrotron_lut.restype = C.c_int
        lib.bh_synchrotron_lut.argtypes = [C.POINTER(SynchrotronLut), vp]
        lib.bh_synchrotron_lut_host.restype = C.c_int
        lib.bh_synchrotron_lut_host.argtypes = [C.POINTER(SynchrotronLut), vp]
        lib.bh_kerr_trace_rt.restype = C.c_int
        lib.bh_kerr_trace_rt.argtypes = [C.POINTER(KerrScene), C.POINTER(GrmhdGrid), C.POINTER(SynchrotronLut),
                                         C.POINTER(RtParams), vp, vp, vp, vp, vp]
        lib.bh_grmhd_packed_read.restype = C.c_int
        lib.bh_grmhd_packed_read.argtypes = [C.c_char_p, C.POINTER(PackedGrmhdInfo), vp, C.c_int64]
        lib.bh_packed_conversion_defaults.restype = None
        lib.bh_packed_conversion_defaults.argtypes = [C.POINTER(PackedConversion)]
        lib.bh_grmhd_from_packed.restype = C.c_int
        lib.bh_grmhd_from_packed.argtypes = [C.POINTER(GrmhdGrid), C.POINTER(PackedGrmhdInfo), vp, vp, C.c_double,
                                             C.POINTER(PackedConversion), vp]
        lib._rt_declared = True
    return lib


def _stream(stream):
    return None if stream is None else (stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def read_packed(json_path, samples: bool = True) -> tuple[PackedGrmhdInfo, np.ndarray | None]:
    """bh_grmhd_packed_read: metadata and (optionally) the float samples
    [n_r][n_theta][n_phi][4] of a nubhlight_pack dataset."""
    lib = _lib()
    info = PackedGrmhdInfo()
    check(lib.bh_grmhd_packed_read(str(json_path).encode(), C.byref(info), None, 0))
    if not samples:
        return info, None
    out = np.empty((info.n_r, info.n_theta, info.n_phi, 4), np.float32)
    check(lib.bh_grmhd_packed_read(str(json_path).encode(), C.byref(info), out.ctypes.data, out.size))
    return info, out


def conversion_defaults(**kw) -> PackedConversion:
    c = PackedConversion()
    _lib().bh_packed_conversion_defaults(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def torus_defaults(**kw) -> TorusParams:
    t = TorusParams()
    _lib().bh_torus_defaults(C.byref(t))
    for k, v in kw.items():
        setattr(t, k, v)
    return t


def rt_defaults(**kw) -> RtParams:
    r = RtParams()
    _lib().bh_rt_defaults(C.byref(r))
    for k, v in kw.items():
        setattr(r, k, v)
    return r


class Medium:
    """The grid (n_e, Theta_e, |B|) on the device and its descriptor: the
    synthetic torus by default, or frames of simulation output
    (``from_packed``)."""

    def __init__(self, n_r=128, n_theta=64, n_phi=64, r_min=2.0, r_max=50.0, torus: TorusParams | None = None,
                 device="cuda", stream=None, synthetic: bool = True):
        self.cells = torch.empty(n_r, n_theta, n_phi, 4, dtype=torch.float32, device=device)
        self.desc = GrmhdGrid(self.cells.data_ptr(), n_r, n_theta, n_phi, 0, r_min, r_max)
        self.torus = torus or torus_defaults()
        if synthetic:
            check(_lib().bh_grmhd_synthetic(C.byref(self.desc), C.byref(self.torus), _stream(stream)))

    @classmethod
    def from_packed(cls, info: PackedGrmhdInfo, left: torch.Tensor, right: torch.Tensor | None = None,
                    alpha: float = 0.0, conversion: PackedConversion | None = None, n_r=128, n_theta=64, n_phi=64,
                    r_min=2.0, r_max=50.0, stream=None) -> "Medium":
        """bh_grmhd_from_packed: the grid resampled from one packed frame (a
        device float32 tensor [n_r][n_theta][n_phi][4]) or the blend of two."""
        m = cls(n_r, n_theta, n_phi, r_min, r_max, device=left.device, synthetic=False)
        conv = conversion or conversion_defaults()
        check(_lib().bh_grmhd_from_packed(C.byref(m.desc), C.byref(info), left.data_ptr(),
                                          None if right is None else right.data_ptr(), alpha, C.byref(conv),
                                          _stream(stream)))
        return m


class Lut:
    """The thermal-synchrotron table on the device and its descriptor."""

    def __init__(self, n_theta=256, n_x=256, theta_range=(0.1, 1000.0), x_range=(1e-4, 1e4), device="cuda",
                 stream=None):
        self.table = torch.empty(n_theta, n_x, dtype=torch.float32, device=device)
        self.desc = SynchrotronLut(self.table.data_ptr(), n_theta, n_x, math.log(theta_range[0]),
                                   math.log(theta_range[1]), math.log(x_range[0]), math.log(x_range[1]))
        check(_lib().bh_synchrotron_lut(C.byref(self.desc), _stream(stream)))

    def host_table(self) -> np.ndarray:
        out = np.empty((self.desc.n_theta, self.desc.n_x), np.float32)
        check(_lib().bh_synchrotron_lut_host(C.byref(self.desc), out.ctypes.data))
        return out


def trace(scene: KerrScene, medium: Medium, lut: Lut, rt: RtParams | None = None, outs: dict | None = None,
          stream=None) -> dict:
    """I_nu, optical depth, class and steps of every pixel (asynchronous)."""
    n = scene.width * scene.height
    dev = medium.cells.device
    if outs is None:
        outs = {"i_nu": torch.empty(n, dtype=torch.float64, device=dev),
                "tau": torch.empty(n, dtype=torch.float64, device=dev),
                "cls": torch.empty(n, dtype=torch.int32, device=dev),
                "steps": torch.empty(n, dtype=torch.int32, device=dev)}
    rt = rt or rt_defaults()
    ptr = lambda k: outs[k].data_ptr() if k in outs else None  # noqa: E731
    check(_lib().bh_kerr_trace_rt(C.byref(scene), C.byref(medium.desc), C.byref(lut.desc), C.byref(rt),
                                  ptr("i_nu"), ptr("tau"), ptr("cls"), ptr("steps"), _stream(stream)))
    return outs
