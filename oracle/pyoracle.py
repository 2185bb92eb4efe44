"""Python binding of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product package never does.

``Oracle`` wraps oracle/_build/libbh_oracle.so (the restatement in
kerr_oracle.hpp). ``RefLib`` wraps oracle/_ref/libbh_ref.so, the reference's
own compiled src/physics/kerr.cpp behind ref_shim.cpp; it exists only where
the reference sources were available at build time.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from blackhole_b200._abi import KerrImageOut, KerrScene, MAX_CROSSINGS

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "libbh_oracle.so"
REF_SO = HERE / "_ref" / "libbh_ref.so"

_vp, _i32, _i64, _f64 = C.c_void_p, C.c_int32, C.c_int64, C.c_double


def build(quiet: bool = True) -> None:
    """Run oracle/Makefile for the restatement (_build). The libraries of
    oracle/_ref are built from the reference's sources by __graft_entry__.build()
    (make REF_SRC=...) and only loaded here when present."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def host_outputs(n: int, maxc: int) -> dict[str, np.ndarray]:
    """Allocate host output arrays for n pixels."""
    out = {
        "cls": np.zeros(n, np.int32),
        "steps": np.zeros(n, np.int32),
        "n_cross": np.zeros(n, np.int32),
        "r_hit": np.zeros((maxc, n), np.float64),
        "phi_hit": np.zeros((maxc, n), np.float64),
        "g": np.zeros((maxc, n), np.float64),
        "flux": np.zeros(n, np.float64),
        "intensity": np.zeros(n, np.float64),
        "theta_inf": np.zeros(n, np.float64),
        "phi_inf": np.zeros(n, np.float64),
    }
    return out


def out_struct(arrs: dict[str, np.ndarray]) -> KerrImageOut:
    o = KerrImageOut()
    for k, v in arrs.items():
        setattr(o, k, v.ctypes.data)
    return o


def default_threads() -> int:
    return max(1, len(os.sched_getaffinity(0)))


class _Base:
    def _trace(self, fn, scene: KerrScene, pix: np.ndarray | None, n: int, threads: int):
        maxc = max(1, min(MAX_CROSSINGS, scene.max_crossings))
        arrs = host_outputs(n, maxc)
        o = out_struct(arrs)
        idx = None if pix is None else np.ascontiguousarray(pix, dtype=np.int64)
        rc = fn(C.byref(scene), n, _ptr(idx), C.byref(o), threads)
        if rc != 0:
            raise RuntimeError(f"oracle trace failed: {rc}")
        return arrs


class Oracle(_Base):
    """The CPU restatement (kerr_oracle.hpp)."""

    def __init__(self, path: Path = ORACLE_SO):
        if not path.exists():
            build()
        self.lib = C.CDLL(str(path))
        L = self.lib
        L.bho_trace_pixels.argtypes = [C.POINTER(KerrScene), _i64, _vp, C.POINTER(KerrImageOut), C.c_int]
        L.bho_trace_alpha_beta.argtypes = [C.POINTER(KerrScene), _i64, _vp, _vp, C.POINTER(KerrImageOut), C.c_int]
        L.bho_trace_pixels_sky.argtypes = [C.POINTER(KerrScene), _i64, _vp, C.POINTER(KerrImageOut), C.c_int, _vp,
                                           C.c_int]
        L.bho_sky_texels.argtypes = [_i64, _vp, _vp, _vp, C.c_int, _vp]
        L.bho_trace_camera.argtypes = [C.POINTER(KerrScene), _vp, _vp, _i64, _vp, C.POINTER(KerrImageOut), _vp,
                                       C.c_int]
        L.bho_trace_paths.argtypes = [C.POINTER(KerrScene), _i64, _vp, _vp, C.c_int, _vp, _vp, C.c_int]
        L.bho_count_rt_ops.argtypes = ([C.POINTER(KerrScene), _i64, _vp, _vp, C.c_int, C.c_int, C.c_int, _f64, _f64,
                                        _vp, C.c_int, C.c_int] + [_f64] * 8 + [_vp])
        L.bho_trace_rt.argtypes = ([C.POINTER(KerrScene), _i64, _vp, _vp, C.c_int, C.c_int, C.c_int, _f64, _f64, _vp,
                                    C.c_int, C.c_int] + [_f64] * 8 + [_vp] * 4 + [C.c_int])
        L.bho_rt_path.restype = _f64
        L.bho_rt_path.argtypes = [_i64, _vp, _vp, _vp]
        L.bho_trace_alpha_beta_ld.argtypes = L.bho_trace_alpha_beta.argtypes
        L.bho_count_ops.argtypes = [C.POINTER(KerrScene), _f64, _f64, _vp, _vp]
        L.bho_count_step_ops.argtypes = [_f64, _f64, _f64, _vp]
        L.bho_kerr_potentials.argtypes = [_i64, _vp, _vp, _f64, _f64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
        L.bho_kerr_step_mino.argtypes = [_i64] + [_vp] * 6 + [_f64, _f64, _vp, _vp, _vp, _vp, _f64, _i32]
        L.bho_kerr_step_mino_f128.argtypes = [_i64] + [_vp] * 6 + [_f64, _f64, _vp, _vp, _vp, _f64, _i32]
        L.bho_kerr_trace_rays.argtypes = ([_i64] + [_vp] * 9 + [_f64] * 5 + [_i32] + [_vp] * 7 + [C.c_int])
        L.bho_kerr_radii.argtypes = [_f64, _f64, _vp]
        L.bho_nt_normalized_flux.restype = _f64
        L.bho_nt_normalized_flux.argtypes = [_f64, _f64]
        L.bho_nt_radiative_efficiency.restype = _f64
        L.bho_nt_radiative_efficiency.argtypes = [_f64]
        L.bho_disk_g.restype = _f64
        L.bho_disk_g.argtypes = [_f64, _f64, _f64]
        L.bho_unit_mass.restype = _f64

    # --- image tracer ------------------------------------------------------
    def trace_pixels(self, scene: KerrScene, pix: np.ndarray | None = None, threads: int | None = None):
        n = scene.width * scene.height if pix is None else len(pix)
        return self._trace(self.lib.bho_trace_pixels, scene, pix, n, threads or default_threads())

    def trace_pixels_sky(self, scene: KerrScene, sky: np.ndarray, pix: np.ndarray | None = None,
                         threads: int | None = None):
        """trace_pixels plus the cubemap sky (uint16 FP16 bits [6][N][N]) on escaped rays."""
        sky = np.ascontiguousarray(sky).view(np.uint16)
        size = int(round((sky.size / 6) ** 0.5))
        fn = lambda sc, n, idx, o, th: self.lib.bho_trace_pixels_sky(sc, n, idx, o, th, _ptr(sky), size)  # noqa: E731
        n = scene.width * scene.height if pix is None else len(pix)
        return self._trace(fn, scene, pix, n, threads or default_threads())

    def trace_camera(self, scene: KerrScene, cam_f64: np.ndarray, cam_i32: np.ndarray, pix: np.ndarray | None = None,
                     threads: int | None = None):
        """Rays of a finite-distance camera (kerr_oracle.hpp Camera): the image
        outputs plus esc_dir [3][n] (unit escape direction, camera-azimuth frame)."""
        n = int(cam_i32[0]) * int(cam_i32[1]) if pix is None else len(pix)
        cf = np.ascontiguousarray(cam_f64, np.float64)
        ci = np.ascontiguousarray(cam_i32, np.int32)
        idx = None if pix is None else np.ascontiguousarray(pix, np.int64)
        maxc = max(1, min(MAX_CROSSINGS, scene.max_crossings))
        arrs = host_outputs(n, maxc)
        o = out_struct(arrs)
        esc = np.zeros((3, n))
        rc = self.lib.bho_trace_camera(C.byref(scene), _ptr(cf), _ptr(ci), n, _ptr(idx), C.byref(o), _ptr(esc),
                                       threads or default_threads())
        if rc != 0:
            raise RuntimeError("oracle camera trace failed")
        arrs["esc_dir"] = esc
        return arrs

    def count_rt_ops(self, scene: KerrScene, cells: np.ndarray, r_range, lut: np.ndarray, log_theta, log_x, nu,
                     length_cm, ds_max, min_transmit, pix: np.ndarray) -> dict:
        """Operation counts of the transfer over the given pixels (counting scalar)."""
        cells = np.ascontiguousarray(cells, np.float32)
        lut = np.ascontiguousarray(lut, np.float32)
        idx = np.ascontiguousarray(pix, np.int64)
        c = np.zeros(9, np.int64)
        self.lib.bho_count_rt_ops(C.byref(scene), len(idx), _ptr(idx), _ptr(cells), cells.shape[0], cells.shape[1],
                                  cells.shape[2], r_range[0], r_range[1], _ptr(lut), lut.shape[0], lut.shape[1],
                                  log_theta[0], log_theta[1], log_x[0], log_x[1], nu, length_cm, ds_max,
                                  min_transmit, _ptr(c))
        return dict(zip(["add", "mul", "div", "sqrt", "trig", "pow", "cmp", "steps", "samples"], c.tolist()))

    def trace_paths(self, scene: KerrScene, alpha, beta, max_points: int, threads: int | None = None):
        """Positions after every RK4 step of rays at (alpha, beta): xyz [n][max][3], counts [n]."""
        al = np.ascontiguousarray(alpha, np.float64)
        be = np.ascontiguousarray(beta, np.float64)
        n = len(al)
        xyz = np.zeros((n, max_points, 3))
        cnt = np.zeros(n, np.int32)
        self.lib.bho_trace_paths(C.byref(scene), n, _ptr(al), _ptr(be), max_points, _ptr(xyz), _ptr(cnt),
                                 threads or default_threads())
        return xyz, cnt

    def trace_rt(self, scene: KerrScene, cells: np.ndarray, r_range, lut: np.ndarray, log_theta, log_x, nu,
                 length_cm, ds_max, min_transmit, pix: np.ndarray | None = None, threads: int | None = None):
        """Along-ray transfer through the grid cells [n_r][n_th][n_ph][4] with table lut [n_lt][n_lx]."""
        cells = np.ascontiguousarray(cells, np.float32)
        lut = np.ascontiguousarray(lut, np.float32)
        n = scene.width * scene.height if pix is None else len(pix)
        idx = None if pix is None else np.ascontiguousarray(pix, np.int64)
        out = {"i_nu": np.zeros(n), "tau": np.zeros(n), "cls": np.zeros(n, np.int32), "steps": np.zeros(n, np.int32)}
        self.lib.bho_trace_rt(C.byref(scene), n, _ptr(idx), _ptr(cells), cells.shape[0], cells.shape[1],
                              cells.shape[2], r_range[0], r_range[1], _ptr(lut), lut.shape[0], lut.shape[1],
                              log_theta[0], log_theta[1], log_x[0], log_x[1], nu, length_cm, ds_max, min_transmit,
                              _ptr(out["i_nu"]), _ptr(out["tau"]), _ptr(out["cls"]), _ptr(out["steps"]),
                              threads or default_threads())
        return out

    def rt_path(self, j, alpha, ds) -> float:
        j, alpha, ds = (np.ascontiguousarray(v, np.float64) for v in (j, alpha, ds))
        return float(self.lib.bho_rt_path(len(j), _ptr(j), _ptr(alpha), _ptr(ds)))

    def sky_texels(self, x, y, z, size: int) -> np.ndarray:
        x, y, z = (np.ascontiguousarray(v, np.float64) for v in (x, y, z))
        out = np.zeros(len(x), np.int64)
        self.lib.bho_sky_texels(len(x), _ptr(x), _ptr(y), _ptr(z), size, _ptr(out))
        return out

    def trace_alpha_beta(self, scene: KerrScene, alpha, beta, threads: int | None = None, long_double=False):
        alpha = np.ascontiguousarray(alpha, np.float64)
        beta = np.ascontiguousarray(beta, np.float64)
        n = len(alpha)
        maxc = max(1, min(MAX_CROSSINGS, scene.max_crossings))
        arrs = host_outputs(n, maxc)
        fn = self.lib.bho_trace_alpha_beta_ld if long_double else self.lib.bho_trace_alpha_beta
        fn(C.byref(scene), n, _ptr(alpha), _ptr(beta), C.byref(out_struct(arrs)), threads or default_threads())
        return arrs

    def count_ops(self, scene: KerrScene, alpha: float, beta: float):
        counts = np.zeros(7, np.int64)
        steps = np.zeros(1, np.int32)
        cls = self.lib.bho_count_ops(C.byref(scene), alpha, beta, _ptr(counts), _ptr(steps))
        keys = ("add", "mul", "div", "sqrt", "trig", "pow", "cmp")
        return cls, int(steps[0]), dict(zip(keys, counts.tolist()))

    def count_step_ops(self, spin=0.9, alpha=3.0, beta=2.0):
        out = np.zeros(14, np.int64)
        self.lib.bho_count_step_ops(spin, alpha, beta, _ptr(out))
        keys = ("add", "mul", "div", "sqrt", "trig", "pow", "cmp")
        return dict(zip(keys, out[:7].tolist())), dict(zip(keys, out[7:].tolist()))

    # --- reference stepper (Part A) ----------------------------------------
    def potentials(self, r, theta, mass, a, e, lz, q):
        return _potentials(self.lib.bho_kerr_potentials, r, theta, mass, a, e, lz, q)

    def step_mino(self, state: dict, mass, a, e, lz, q, dlam, nsteps=1):
        return _step(self.lib.bho_kerr_step_mino, state, mass, a, e, lz, q, dlam, nsteps)

    def step_mino_f128(self, state: dict, mass, a, e, lz, q, dlam: float, nsteps=1):
        s = {k: np.array(v, np.float64, copy=True) for k, v in state.items()}
        n = len(s["r"])
        args = [_ptr(s[k]) for k in ("r", "theta", "phi", "t", "sign_r", "sign_theta")]
        self.lib.bho_kerr_step_mino_f128(n, *args, mass, a, _ptr(np.asarray(e, np.float64)),
                                         _ptr(np.asarray(lz, np.float64)), _ptr(np.asarray(q, np.float64)),
                                         dlam, nsteps)
        return s

    def trace_rays(self, state, e, lz, q, mass, a, r_horizon, r_escape, step, max_steps, threads=None):
        return _trace_rays(self.lib.bho_kerr_trace_rays, state, e, lz, q, mass, a, r_horizon, r_escape,
                           step, max_steps, threads or default_threads())

    def radii(self, m: float, a: float):
        out = np.zeros(8, np.float64)
        self.lib.bho_kerr_radii(m, a, _ptr(out))
        keys = ("r_plus", "r_minus", "isco_pro", "isco_retro", "r_ph_pro", "r_ph_retro", "nt_isco", "nt_peak")
        return dict(zip(keys, out.tolist()))

    def nt_flux(self, r: float, a_star: float) -> float:
        return self.lib.bho_nt_normalized_flux(r, a_star)

    def nt_efficiency(self, a_star: float) -> float:
        return self.lib.bho_nt_radiative_efficiency(a_star)

    def disk_g(self, r: float, a: float, lam: float) -> float:
        return self.lib.bho_disk_g(r, a, lam)

    @property
    def unit_mass(self) -> float:
        return self.lib.bho_unit_mass()


class RefLib(_Base):
    """The reference's own compiled kerr.cpp behind ref_shim.cpp."""

    def __init__(self, path: Path = REF_SO):
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (reference sources absent at build time)")
        self.lib = C.CDLL(str(path))
        L = self.lib
        for fn in ("ref_synchrotron_j", "ref_synchrotron_alpha"):
            getattr(L, fn).restype = _f64
            getattr(L, fn).argtypes = [_f64] * 4
        L.ref_planck.restype = _f64
        L.ref_planck.argtypes = [_f64, _f64]
        L.ref_rte_path.restype = _f64
        L.ref_rte_path.argtypes = [_i64, _vp, _vp, _vp]
        L.ref_kerr_potentials.argtypes = [_i64, _vp, _vp, _f64, _f64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
        L.ref_kerr_step_mino.argtypes = [_i64] + [_vp] * 6 + [_f64, _f64, _vp, _vp, _vp, _vp, _f64, _i32]
        L.ref_kerr_trace_rays.argtypes = ([_i64] + [_vp] * 9 + [_f64] * 5 + [_i32] + [_vp] * 7 + [C.c_int])
        L.ref_kerr_raytracer_defaults.argtypes = [_f64, _f64, _vp]
        L.ref_trace_pixels.argtypes = [C.POINTER(KerrScene), _i64, _vp, C.POINTER(KerrImageOut), C.c_int]
        L.ref_kerr_radii.argtypes = [_f64, _f64, _vp]
        L.ref_nt_normalized_flux.restype = _f64
        L.ref_nt_normalized_flux.argtypes = [_f64, _f64]

    @staticmethod
    def available() -> bool:
        return REF_SO.exists()

    def potentials(self, r, theta, mass, a, e, lz, q):
        return _potentials(self.lib.ref_kerr_potentials, r, theta, mass, a, e, lz, q)

    def step_mino(self, state: dict, mass, a, e, lz, q, dlam, nsteps=1):
        return _step(self.lib.ref_kerr_step_mino, state, mass, a, e, lz, q, dlam, nsteps)

    def trace_rays(self, state, e, lz, q, mass, a, r_horizon, r_escape, step, max_steps, threads=None):
        return _trace_rays(self.lib.ref_kerr_trace_rays, state, e, lz, q, mass, a, r_horizon, r_escape,
                           step, max_steps, threads or default_threads())

    def synchrotron_j(self, nu, b, n, theta):
        return self.lib.ref_synchrotron_j(nu, b, n, theta)

    def synchrotron_alpha(self, nu, b, n, theta):
        return self.lib.ref_synchrotron_alpha(nu, b, n, theta)

    def planck(self, nu, temp):
        return self.lib.ref_planck(nu, temp)

    def rte_path(self, j, alpha, ds) -> float:
        j, alpha, ds = (np.ascontiguousarray(v, np.float64) for v in (j, alpha, ds))
        return float(self.lib.ref_rte_path(len(j), _ptr(j), _ptr(alpha), _ptr(ds)))

    def raytracer_defaults(self, mass: float, spin_param: float):
        out = np.zeros(4, np.float64)
        self.lib.ref_kerr_raytracer_defaults(mass, spin_param, _ptr(out))
        return dict(a=out[0], r_horizon=out[1], r_escape=out[2], step_size=out[3])

    def trace_pixels(self, scene: KerrScene, pix: np.ndarray | None = None, threads: int | None = None):
        n = scene.width * scene.height if pix is None else len(pix)
        return self._trace(self.lib.ref_trace_pixels, scene, pix, n, threads or default_threads())

    def radii(self, mass: float, a: float):
        out = np.zeros(10, np.float64)
        self.lib.ref_kerr_radii(mass, a, _ptr(out))
        keys = ("r_plus", "r_minus", "isco_pro", "isco_retro", "r_ph_pro", "r_ph_retro",
                "nt_isco", "nt_efficiency", "nt_flux_peak", "nt_flux_10")
        return dict(zip(keys, out.tolist()))

    def nt_flux(self, r: float, a_star: float) -> float:
        return self.lib.ref_nt_normalized_flux(r, a_star)


def _potentials(fn, r, theta, mass, a, e, lz, q):
    r = np.ascontiguousarray(r, np.float64)
    n = len(r)
    outs = [np.zeros(n) for _ in range(4)]
    fn(n, _ptr(r), _ptr(np.ascontiguousarray(theta, np.float64)), mass, a,
       _ptr(np.ascontiguousarray(e, np.float64)), _ptr(np.ascontiguousarray(lz, np.float64)),
       _ptr(np.ascontiguousarray(q, np.float64)), *[_ptr(o) for o in outs])
    return dict(zip(("r_pot", "dr_pot", "theta_pot", "dtheta_pot"), outs))


def _step(fn, state, mass, a, e, lz, q, dlam, nsteps):
    s = {k: np.array(v, np.float64, copy=True) for k, v in state.items()}
    n = len(s["r"])
    args = [_ptr(s[k]) for k in ("r", "theta", "phi", "t", "sign_r", "sign_theta")]
    if np.ndim(dlam) == 0:
        dl, scalar = None, float(dlam)
    else:
        dl, scalar = np.ascontiguousarray(dlam, np.float64), 0.0
    fn(n, *args, mass, a, _ptr(np.ascontiguousarray(e, np.float64)), _ptr(np.ascontiguousarray(lz, np.float64)),
       _ptr(np.ascontiguousarray(q, np.float64)), _ptr(dl), scalar, nsteps)
    return s


def _trace_rays(fn, state, e, lz, q, mass, a, r_horizon, r_escape, step, max_steps, threads):
    n = len(state["r"])
    ins = [np.ascontiguousarray(state[k], np.float64) for k in ("r", "theta", "phi", "t", "sign_r", "sign_theta")]
    cs = [np.ascontiguousarray(x, np.float64) for x in (e, lz, q)]
    st = np.zeros(n, np.int32)
    steps = np.zeros(n, np.int32)
    fl = [np.zeros(n) for _ in range(5)]
    fn(n, *[_ptr(x) for x in ins], *[_ptr(x) for x in cs], mass, a, r_horizon, r_escape, step, max_steps,
       _ptr(st), _ptr(steps), *[_ptr(x) for x in fl], threads)
    return dict(status=st, steps=steps, total_distance=fl[0], r=fl[1], theta=fl[2], phi=fl[3], redshift=fl[4])
