"""ctypes mirror of the C ABI in include/bh_kerr.h and the library loader.

The CUDA library ``blackhole_b200/lib/libblackhole_b200.so`` is built in-tree
(``python -m blackhole_b200.build`` or ``__graft_entry__.build()``). Loading
fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "lib" / "libblackhole_b200.so"

# enum BH_PixelClass
CLASS_CAPTURED, CLASS_DISK, CLASS_ESCAPED, CLASS_MAX_STEPS = 0, 1, 2, 3
# enum BH_Integrator
INTEGRATOR_RK4, INTEGRATOR_DP45, INTEGRATOR_ANALYTIC = 0, 1, 2
# enum BH_Precision
PRECISION_FP64, PRECISION_MIXED = 0, 1
# enum BH_PotentialForm
POTENTIAL_REFERENCE, POTENTIAL_CARTER = 0, 1
# enum BH_RayStatus (physics::RayStatus)
STATUS_PROPAGATING, STATUS_ESCAPED, STATUS_CAPTURED, STATUS_HIT_DISK, STATUS_MAX_STEPS = 0, 1, 2, 3, 4
MAX_CROSSINGS = 3


class KerrScene(C.Structure):
    """struct BH_KerrScene."""

    _fields_ = [
        ("spin", C.c_double),
        ("r_obs", C.c_double),
        ("theta_obs", C.c_double),
        ("alpha_min", C.c_double),
        ("alpha_max", C.c_double),
        ("beta_min", C.c_double),
        ("beta_max", C.c_double),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("integrator", C.c_int32),
        ("precision", C.c_int32),
        ("potential_form", C.c_int32),
        ("max_crossings", C.c_int32),
        ("max_steps", C.c_int32),
        ("reserved0", C.c_int32),
        ("step_coeff", C.c_double),
        ("step_rcap", C.c_double),
        ("rtol", C.c_double),
        ("atol", C.c_double),
        ("horizon_factor", C.c_double),
        ("escape_factor", C.c_double),
        ("disk_r_in", C.c_double),
        ("disk_r_out", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved0"}


class KerrImageOut(C.Structure):
    """struct BH_KerrImageOut (all pointers; NULL = not wanted)."""

    _fields_ = [
        ("cls", C.c_void_p),
        ("steps", C.c_void_p),
        ("n_cross", C.c_void_p),
        ("r_hit", C.c_void_p),
        ("phi_hit", C.c_void_p),
        ("g", C.c_void_p),
        ("flux", C.c_void_p),
        ("intensity", C.c_void_p),
        ("theta_inf", C.c_void_p),
        ("phi_inf", C.c_void_p),
        ("carter_drift", C.c_void_p),
    ]


class KerrStateSoA(C.Structure):
    """struct BH_KerrStateSoA (device pointers)."""

    _fields_ = [(n, C.c_void_p) for n in ("r", "theta", "phi", "t", "sign_r", "sign_theta")]


class KerrConstsSoA(C.Structure):
    """struct BH_KerrConstsSoA (device pointers)."""

    _fields_ = [(n, C.c_void_p) for n in ("e", "lz", "q")]


class KerrRaytracerParams(C.Structure):
    """struct BH_KerrRaytracerParams."""

    _fields_ = [
        ("mass", C.c_double),
        ("a", C.c_double),
        ("r_horizon", C.c_double),
        ("r_escape", C.c_double),
        ("step_size", C.c_double),
        ("max_steps", C.c_int32),
        ("reserved", C.c_int32),
    ]


class KerrLaunchConfig(C.Structure):
    """struct BH_KerrLaunchConfig."""

    _fields_ = [("block_threads", C.c_int32), ("ctas_per_sm", C.c_int32), ("refill_steps", C.c_int32),
                ("reserved", C.c_int32)]


class SkyCubemap(C.Structure):
    """struct BH_SkyCubemap (device FP16 texels [6][size][size])."""

    _fields_ = [("texels", C.c_void_p), ("size", C.c_int32), ("reserved", C.c_int32)]


class AdamConfig(C.Structure):
    """struct BH_AdamConfig."""

    _fields_ = [("lr", C.c_float), ("beta1", C.c_float), ("beta2", C.c_float), ("eps", C.c_float)]


class SurrogatePolicy(C.Structure):
    """struct BH_SurrogatePolicy."""

    _fields_ = [("min_confidence", C.c_float), ("verify", C.c_int32), ("critical_band", C.c_double),
                ("refine_fp64", C.c_int32), ("chunks", C.c_int32)]


class SurrogateStats(C.Structure):
    """struct BH_SurrogateStats."""

    _fields_ = [(n, C.c_int64) for n in ("pixels", "accepted", "low_confidence", "critical_band", "solve_failed",
                                         "disagreement")]


# the ten standard fields (carter_drift, the mixed tracer's diagnostic, is asked for by name)
OUT_FIELDS = [name for name, _ in KerrImageOut._fields_ if name != "carter_drift"]
# carter_drift is a diagnostic the device entry points write on request only.
DEVICE_OUT_FIELDS = [name for name, _ in KerrImageOut._fields_]
INT_FIELDS = ("cls", "steps", "n_cross")
PLANE_FIELDS = ("r_hit", "phi_hit", "g")


def default_scene(**overrides) -> KerrScene:
    """The 256x256 a=0.9 thin-disk scene (observer r=1000, 60 deg), overridable."""
    s = KerrScene()
    s.spin = 0.9
    s.r_obs = 1000.0
    s.theta_obs = 60.0 * 3.141592653589793 / 180.0
    s.alpha_min, s.alpha_max = -12.0, 12.0
    s.beta_min, s.beta_max = -12.0, 12.0
    s.width = s.height = 256
    s.integrator = INTEGRATOR_RK4
    s.precision = PRECISION_FP64
    s.potential_form = POTENTIAL_REFERENCE
    s.max_crossings = 1
    s.max_steps = 20000
    s.step_coeff = 0.02
    s.step_rcap = 20.0
    s.rtol = 1e-8
    s.atol = 1e-10
    s.horizon_factor = 1.001
    s.escape_factor = 1.01
    s.disk_r_in = 0.0
    s.disk_r_out = 30.0
    for k, v in overrides.items():
        if not hasattr(s, k):
            raise AttributeError(f"BH_KerrScene has no field {k!r}")
        setattr(s, k, v)
    return s


_LIB = None


def load_library() -> C.CDLL:
    """Load the CUDA library (once). Raises if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = Path(os.environ.get("BH_B200_LIB", LIB_PATH))
    if not path.exists():
        raise RuntimeError(
            f"{path} is missing: build the CUDA library first "
            "(python -m blackhole_b200.build). There is no CPU fallback."
        )
    lib = C.CDLL(str(path))
    _declare(lib)
    _LIB = lib
    return lib


def _declare(lib: C.CDLL) -> None:
    vp, i32, i64, f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    lib.bh_last_error.restype = C.c_char_p
    lib.bh_last_error.argtypes = []
    lib.bh_abi_version.restype = C.c_int
    lib.bh_kerr_potentials.restype = C.c_int
    lib.bh_kerr_potentials.argtypes = [i64, vp, vp, f64, f64, KerrConstsSoA, vp, vp, vp, vp, vp]
    lib.bh_kerr_step_mino.restype = C.c_int
    lib.bh_kerr_step_mino.argtypes = [i64, KerrStateSoA, f64, f64, KerrConstsSoA, vp, f64, vp]
    lib.bh_kerr_raytracer_defaults.restype = C.c_int
    lib.bh_kerr_raytracer_defaults.argtypes = [f64, f64, C.POINTER(KerrRaytracerParams)]
    lib.bh_kerr_trace_rays.restype = C.c_int
    lib.bh_kerr_trace_rays.argtypes = [
        i64, KerrStateSoA, KerrConstsSoA, C.POINTER(KerrRaytracerParams),
        vp, vp, vp, vp, vp, vp, vp, vp,
    ]
    lib.bh_kerr_scene_defaults.restype = None
    lib.bh_kerr_scene_defaults.argtypes = [C.POINTER(KerrScene)]
    lib.bh_kerr_scene_validate.restype = C.c_int
    lib.bh_kerr_scene_validate.argtypes = [C.POINTER(KerrScene)]
    lib.bh_kerr_trace_image.restype = C.c_int
    lib.bh_kerr_trace_image.argtypes = [C.POINTER(KerrScene), C.POINTER(KerrImageOut), vp]
    lib.bh_kerr_trace_image_host.restype = C.c_int
    lib.bh_kerr_trace_image_host.argtypes = [C.POINTER(KerrScene), C.POINTER(KerrImageOut)]
    lib.bh_kerr_set_launch.restype = C.c_int
    lib.bh_kerr_set_launch.argtypes = [i32, i32]
    lib.bh_kerr_trace_image_host_noalloc.restype = C.c_int
    lib.bh_kerr_trace_image_host_noalloc.argtypes = [C.POINTER(KerrScene), C.POINTER(KerrImageOut), vp]
    lib.bh_kerr_batch_create.restype = vp
    lib.bh_kerr_batch_create.argtypes = [C.POINTER(KerrScene), C.POINTER(KerrImageOut), i32]
    for fn in ("bh_kerr_batch_trace", "bh_kerr_batch_trace_graph"):
        getattr(lib, fn).restype = C.c_int
        getattr(lib, fn).argtypes = [vp, vp]
    lib.bh_kerr_batch_set_launch.restype = C.c_int
    lib.bh_kerr_batch_set_launch.argtypes = [vp, C.POINTER(KerrLaunchConfig)]
    lib.bh_kerr_batch_get_launch.restype = C.c_int
    lib.bh_kerr_batch_get_launch.argtypes = [vp, C.POINTER(KerrLaunchConfig)]
    lib.bh_kerr_batch_autotune.restype = C.c_int
    lib.bh_kerr_batch_autotune.argtypes = [vp, i64, vp, C.POINTER(KerrLaunchConfig)]
    lib.bh_kerr_batch_frame_times.restype = C.c_int
    lib.bh_kerr_batch_frame_times.argtypes = [vp, vp]
    lib.bh_kerr_batch_frames.restype = i32
    lib.bh_kerr_batch_frames.argtypes = [vp]
    lib.bh_kerr_batch_pixels.restype = i64
    lib.bh_kerr_batch_pixels.argtypes = [vp]
    lib.bh_kerr_batch_destroy.restype = None
    lib.bh_kerr_batch_destroy.argtypes = [vp]
    lib.bh_sky_generate.restype = C.c_int
    lib.bh_sky_generate.argtypes = [vp, i32, i32, C.c_uint64, vp]
    lib.bh_kerr_trace_image_sky.restype = C.c_int
    lib.bh_kerr_trace_image_sky.argtypes = [C.POINTER(KerrScene), C.POINTER(KerrImageOut), C.POINTER(SkyCubemap), vp]
    lib.bh_kerr_batch_set_sky.restype = C.c_int
    lib.bh_kerr_batch_set_sky.argtypes = [vp, C.POINTER(SkyCubemap)]
    lib.bh_debug_device_allocations.restype = C.c_int64
    lib.bh_debug_device_allocations.argtypes = []
    lib.bh_debug_fail_device_allocation.restype = C.c_int
    lib.bh_debug_fail_device_allocation.argtypes = [C.c_int64]
    # include/bh_surrogate.h
    lib.bh_surrogate_param_count.restype = i64
    lib.bh_surrogate_param_count.argtypes = []
    lib.bh_surrogate_create.restype = vp
    lib.bh_surrogate_create.argtypes = [i64, C.c_uint64]
    lib.bh_surrogate_destroy.restype = None
    lib.bh_surrogate_destroy.argtypes = [vp]
    for fn in ("bh_surrogate_get_params", "bh_surrogate_set_params"):
        getattr(lib, fn).restype = C.c_int
        getattr(lib, fn).argtypes = [vp, vp, i64]
    lib.bh_surrogate_features.restype = C.c_int
    lib.bh_surrogate_features.argtypes = [vp, i64, vp, vp]
    lib.bh_surrogate_forward.restype = C.c_int
    lib.bh_surrogate_forward.argtypes = [vp, vp, i64, vp, vp]
    lib.bh_surrogate_gradients.restype = C.c_int
    lib.bh_surrogate_gradients.argtypes = [vp, vp, vp, i64, vp, vp, vp]
    lib.bh_surrogate_train_step.restype = C.c_int
    lib.bh_surrogate_train_step.argtypes = [vp, vp, vp, i64, C.POINTER(AdamConfig), vp, vp]
    lib.bh_surrogate_device_error.restype = C.c_int
    lib.bh_surrogate_device_error.argtypes = [vp]
    lib.bh_surrogate_get_state.restype = C.c_int
    lib.bh_surrogate_get_state.argtypes = [vp, vp, vp, C.c_int64, C.POINTER(C.c_int64)]
    lib.bh_surrogate_set_state.restype = C.c_int
    lib.bh_surrogate_set_state.argtypes = [vp, vp, vp, C.c_int64, C.c_int64]
    lib.bh_surrogate_set_wait_limit.restype = C.c_int
    lib.bh_surrogate_set_wait_limit.argtypes = [vp, C.c_int64]
    lib.bh_surrogate_make_targets.restype = C.c_int
    lib.bh_surrogate_make_targets.argtypes = [C.POINTER(KerrImageOut), i64, C.c_int, vp, vp]
    lib.bh_surrogate_grid_inputs.restype = C.c_int
    lib.bh_surrogate_grid_inputs.argtypes = [C.POINTER(KerrScene), vp, vp]
    lib.bh_surrogate_policy_defaults.restype = None
    lib.bh_surrogate_policy_defaults.argtypes = [C.POINTER(SurrogatePolicy)]
    lib.bh_surrogate_trace_image.restype = C.c_int
    lib.bh_surrogate_trace_image.argtypes = [vp, C.POINTER(KerrScene), C.POINTER(KerrImageOut),
                                             C.POINTER(SurrogatePolicy), vp]
    lib.bh_surrogate_trace_image_host.restype = C.c_int
    lib.bh_surrogate_trace_image_host.argtypes = [vp, C.POINTER(KerrScene), C.POINTER(KerrImageOut),
                                                  C.POINTER(SurrogatePolicy)]
    lib.bh_surrogate_last_stats.restype = C.c_int
    lib.bh_surrogate_last_stats.argtypes = [vp, C.POINTER(SurrogateStats)]
    lib.bh_bf16_gemm.restype = C.c_int
    lib.bh_bf16_gemm.argtypes = [vp, vp, i64, C.c_int, C.c_int, vp, vp]


def check(rc: int) -> None:
    """Raise RuntimeError with bh_last_error() when a C call returned non-zero."""
    if rc != 0:
        msg = load_library().bh_last_error().decode("utf-8", "replace")
        raise RuntimeError(msg or f"blackhole_b200 call failed with code {rc}")
