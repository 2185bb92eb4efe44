"""Benchmark: Kerr rays/s on one B200 (or N independent replicas).

Default workload ``c4_2048``: the a = 0.9 thin-disk scene (observer at
r = 1000 M, 60 deg, alpha, beta in [-12, 12] M, opaque disk r_isco..30 M)
at 2048 x 2048 pixels rendered by mixed precision plus the learned
surrogate (bh_surrogate_trace_image: network inference on every pixel,
exact Mino-time refinement, the closed-form tracer on rejected pixels and
the mixed DP45 integrator on the few it does not cover),
beside the plain FP64 integrators on the same scene: FP64 DP45 (rtol 1e-8)
at 2048^2 and FP64 RK4 with h = 0.02 min(r, 20) (the plain method of the
256^2 scene) timed on its 256^2 frame. One step = one render of the frame.

Other workloads (``--workload``): ``disk16`` (16 frames of 1024^2, spins
{0, 0.5, 0.9, 0.998} x inclinations {17, 45, 75, 85} deg, DP45, 3 crossings,
one persistent launch), ``batch4096`` (4096 uneven frames in one launch),
single frames ``c0_256``, ``disk1_512``, ``disk1_1024``, ``disk_2048``.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun as N independent replicas (every pixel is
independent: no exchange step); value = all ranks' rays / max-over-ranks time.
``--impl reference`` times the reference's own CPU path on the host cores
(oracle/_ref: the reference's compiled src/physics/kerr.cpp potentials
driving the same tracer) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Kerr rays/sec on 1 B200: FP64 plain vs mixed/surrogate at stated g-error"
UNIT = "rays/s"

# Algorithmic FLOPs (add, mul, div, sqrt each 1) per accepted integration
# step, frozen from the oracle's counting scalar over seeded pixels of each
# workload (tests/test_flop_constants.py re-derives them). The mixed path runs
# the same algorithm, so the same count applies to it. "rt": one accepted DP45
# step of the volumetric transfer (c2_512) with its medium samples (2.1 per
# step on average; exp/log/acos not counted as FLOPs).
FLOPS_PER_STEP = {"dp45": 506.0, "rk4": 213.0, "rt": 1001.0}

# DRAM bytes (read + write) of one k_mlp_infer launch on the 2048^2 frame,
# from one single-pass ncu capture of this script's default run
# (profiles/k_mlp_infer_c4_1024.md gives the command): 67.8 MB read (inputs and
# weights), 214.6 MB written (the rest of the 268 MB of outputs is still in L2
# when the kernel ends).
INFER_DRAM_BYTES_2048 = 67833856 + 214636288

WORKLOADS = {
    # name: (frames, width, integrator, max_crossings)
    "disk16": dict(width=1024, height=1024, integrator=1, max_crossings=3, sky=True,
                   frames=[(a, i) for a in (0.0, 0.5, 0.9, 0.998) for i in (17.0, 45.0, 75.0, 85.0)]),
    "c0_256": dict(width=256, height=256, integrator=0, max_crossings=1, frames=[(0.9, 60.0)]),
    "disk1_512": dict(width=512, height=512, integrator=1, max_crossings=3, frames=[(0.9, 45.0)]),
    "disk1_1024": dict(width=1024, height=1024, integrator=1, max_crossings=3, frames=[(0.9, 45.0)]),
    "disk_2048": dict(width=2048, height=2048, integrator=0, max_crossings=1, frames=[(0.9, 60.0)]),
    "batch4096": dict(integrator=1, max_crossings=1, generator=lambda: batch_frames()),
    "c4_2048": dict(width=2048, height=2048, integrator=1, max_crossings=1, frames=[(0.9, 60.0)], surrogate=True),
    "c2_512": dict(width=512, height=512, integrator=1, max_crossings=1, frames=[(0.94, 17.0)], rt=True),
    # smaller copies of the two scenes above, for profiler captures
    "c4_1024": dict(width=1024, height=1024, integrator=1, max_crossings=1, frames=[(0.9, 60.0)], surrogate=True),
    # the closed-form tracer (BH_INTEGRATOR_ANALYTIC, FP64) on the C4 frame, and a
    # 512^2 three-crossing frame for profiler captures
    "c4_analytic": dict(width=2048, height=2048, integrator=2, max_crossings=1, frames=[(0.9, 60.0)], analytic=True),
    "disk1_512_analytic": dict(width=512, height=512, integrator=2, max_crossings=3, frames=[(0.9, 45.0)],
                               analytic=True),
    "disk1_1024_analytic": dict(width=1024, height=1024, integrator=2, max_crossings=3, frames=[(0.9, 45.0)],
                                analytic=True),
    "c2_128": dict(width=128, height=128, integrator=1, max_crossings=1, frames=[(0.94, 17.0)], rt=True),
}
SURROGATE_WEIGHTS = ROOT / "blackhole_b200" / "data" / "surrogate_c4.npz"
# The sky of escaping rays in the disk16 workload: 6 x 512 x 512 FP16 cubemap,
# seeded uniform noise plus 10^4 point stars (bh_sky_generate).
SKY_SIZE, SKY_STARS, SKY_SEED = 512, 10_000, 20261203
# Algorithmic MACs per ray of the network, 2 FLOPs each: 134 input features
# (128 Fourier, 4 raw inputs, lambda, eta) x 256, 3 x 256 x 256, 256 x 16
# heads. The kernel executes the input layer on 144 columns (two 64-column
# K chunks and the one 16-column K step of the third that holds features
# 128..133): SURROGATE_MMA_FLOPS_PER_RAY.
SURROGATE_FLOPS_PER_RAY = 2.0 * (134 * 256 + 3 * 256 * 256 + 256 * 16)
SURROGATE_MMA_FLOPS_PER_RAY = 2.0 * (144 * 256 + 3 * 256 * 256 + 256 * 16)
OUT_FIELDS_USED = ("cls", "steps", "n_cross", "r_hit", "phi_hit", "g", "flux", "intensity", "theta_inf", "phi_inf")


CARTER_DRIFT_DEF = ("largest relative residual |eta(state) - eta| / (|q_Th| + a^2) that the tracer's projection "
                    "removed from a ray (BH_KerrImageOut.carter_drift), over the frame; 0 for solved pixels")


def carter_drift_stats(trace, n: int, device) -> dict:
    """Carter-constant drift of one untimed render: ``trace(outs)`` writes the
    frame's steps and carter_drift into ``outs``."""
    import torch

    outs = {"steps": torch.empty(n, dtype=torch.int32, device=device),
            "carter_drift": torch.empty(n, dtype=torch.float64, device=device)}
    trace(outs)
    torch.cuda.synchronize(device)
    d = outs["carter_drift"]
    stepped = outs["steps"] > 0
    ds = d[stepped]
    return {"max": float(d.max().item()),
            "median_stepped": float(ds.median().item()) if ds.numel() else 0.0,
            "p99_stepped": float(torch.quantile(ds[:1 << 24].float(), 0.99).item()) if ds.numel() else 0.0,
            "stepped_pixels": int(stepped.sum().item())}


def fma_probe():
    """The bench's FMA-pipe peak probe (blackhole_b200/lib/libbh_bench_probe.so,
    built beside the tracer library but not part of it)."""
    lib = C.CDLL(str(ROOT / "blackhole_b200" / "lib" / "libbh_bench_probe.so"))
    lib.bh_bench_fma_peak.restype = C.c_int
    lib.bh_bench_fma_peak.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double)]
    return lib


def _check_probe(rc: int) -> None:
    if rc != 0:
        raise RuntimeError("bh_bench_fma_peak failed")


def batch_frames(n: int = 4096, seed: int = 20261203):
    """The uneven batch: per frame (own seed) a size from {64, 128, 256, 512}^2,
    a ~ U[0, 0.998], inclination ~ U[5, 89] deg, r_obs ~ logU[100, 5000] M."""
    frames = []
    for i in range(n):
        rng = np.random.default_rng([seed, i])
        side = int(rng.choice([64, 128, 256, 512]))
        frames.append(dict(width=side, height=side, spin=float(rng.uniform(0.0, 0.998)),
                           theta_obs=math.radians(float(rng.uniform(5.0, 89.0))),
                           r_obs=float(math.exp(rng.uniform(math.log(100.0), math.log(5000.0))))))
    return frames


def scenes_for(workload: str, precision: int):
    from blackhole_b200._abi import default_scene

    w = WORKLOADS[workload]
    if "generator" in w:
        return [default_scene(integrator=w["integrator"], max_crossings=w["max_crossings"], precision=precision, **f)
                for f in w["generator"]()]
    out = []
    for spin, inc in w["frames"]:
        out.append(default_scene(width=w["width"], height=w["height"], spin=spin, theta_obs=math.radians(inc),
                                 integrator=w["integrator"], max_crossings=w["max_crossings"],
                                 precision=precision))
    return out


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock, its maximum, power and the throttle reasons of one GPU,
    polled through NVML every 5 ms from a thread (reads only)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples: list[tuple] = []
        self._stop = threading.Event()
        self._on = threading.Event()
        self._t = None
        self.nvml = None

    def start(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.sm_max = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nvml = None
            return
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        p = self.nvml
        while not self._stop.is_set():
            if self._on.is_set():
                try:
                    sm = p.nvmlDeviceGetClockInfo(self.h, p.NVML_CLOCK_SM)
                    reasons = p.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                    power = p.nvmlDeviceGetPowerUsage(self.h) / 1000.0
                    self.samples.append((sm, reasons, power))
                except Exception:
                    pass
            time.sleep(0.005)

    def wait_first_sample(self, timeout_s: float = 5.0) -> None:
        """Arm the sampler (call just before the timed region)."""
        self.samples.clear()
        self._on.set()

    @property
    def lines(self):
        return self.samples

    def stop(self) -> dict:
        if self.nvml is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["NVML unavailable"]}
        time.sleep(0.012)  # at least one more sample after the timed region
        self._on.clear()
        self._stop.set()
        if self._t is not None:
            self._t.join(timeout=1.0)
        sm = [s[0] for s in self.samples]
        reasons = sorted(name for name, bit in self.REASONS.items() if any(s[1] & bit for s in self.samples))
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.sm_max, "reasons": reasons,
                "samples": len(sm), "power_w_max": max((s[2] for s in self.samples), default=None),
                "source": "NVML, 5 ms polling during the timed region"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def time_precision(args, precision: str, dev, stream, dist):
    """Warm up, then time ``args.steps`` renders of the workload at one precision."""
    import torch

    from blackhole_b200 import kerr

    scenes = scenes_for(args.workload, 1 if precision == "mixed" else 0)
    # All frames of a step go out as one persistent launch, replayed from a
    # CUDA graph; the per-step events bracket that one launch.
    batch = kerr.TraceBatch(scenes, device=dev, fields=list(OUT_FIELDS_USED))
    if WORKLOADS[args.workload].get("sky"):
        batch.set_sky(kerr.sky_generate(SKY_SIZE, SKY_STARS, SKY_SEED, device=dev))
    outs = batch.outs
    tuned = batch.autotune(stream=stream) if args.autotune else batch.launch()

    def render(ev=None):
        if ev is not None:
            ev[0][0].record(stream)
        batch.trace_graph(stream=stream)
        if ev is not None:
            ev[0][1].record(stream)

    sampler = ClockSampler(dev.index if "CUDA_VISIBLE_DEVICES" not in os.environ else 0)
    sampler.start()
    sampler.wait_first_sample()
    for _ in range(args.warmup):
        render()
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    sampler.lines.clear()
    per_launch = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))]
                  for _ in range(args.steps)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(args.steps):
        render(per_launch[k])
    t1.record(stream)
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    if dist is not None:
        dist.barrier()
    elapsed_ms = t0.elapsed_time(t1)
    if dist is not None:
        t = torch.tensor([elapsed_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    launch_ms = [a.elapsed_time(b) for step in per_launch for (a, b) in step]
    total_steps = sum(int(o["steps"].sum().item()) for o in outs)  # accepted steps of one render
    frame_ms = batch.frame_times()  # completion of each frame within the last launch
    return dict(scenes=scenes, outs=outs, elapsed_ms=elapsed_ms, launch_ms=launch_ms, total_steps=total_steps,
                clocks=clocks, frame_ms=frame_ms, launch_cfg=tuned, batch=batch)


def _stats(x, unit: str) -> dict:
    """Median, 99.9th percentile and maximum of a 1-D tensor of errors."""
    import torch

    if x.numel() == 0:
        return {"median": None, "p999": None, "max": None, "n": 0, "unit": unit}
    xs = x.double()
    q = torch.quantile(xs[:16_000_000], torch.tensor([0.5, 0.999], dtype=torch.float64, device=xs.device)).tolist()
    return {"median": q[0], "p999": q[1], "max": float(xs.max().item()), "n": int(xs.numel()), "unit": unit}


def _wrap_abs(d):
    """|d| reduced modulo 2 pi into [0, pi] (azimuths are angles)."""
    import torch

    return torch.remainder(d + math.pi, 2.0 * math.pi).sub(math.pi).abs()


def accuracy(ref_outs, test_outs, reference: str = "this run's FP64 path (bit-identical to the CPU oracle)") -> dict:
    """Errors of ``test`` against ``ref`` over all frames. Class agreement over
    every pixel; the other fields on pixels whose class (and, for disk
    fields, crossing count) agree: r_hit and g relative at every crossing,
    phi_hit in radians modulo 2 pi, flux and intensity absolute in units of
    the frame's peak (the flux vanishes at the ISCO, so a relative error
    there says nothing), theta_inf and phi_inf in radians on escaped pixels.
    The legacy keys dg_over_g_* are g at the last recorded crossing."""
    import torch

    agree = total = 0
    dgs = []
    errs = {k: [] for k in ("r_hit", "g", "phi_hit", "flux", "intensity", "theta_inf", "phi_inf")}
    for a, b in zip(ref_outs, test_outs):
        same_cls = a["cls"] == b["cls"]
        agree += int(same_cls.sum().item())
        total += a["cls"].numel()
        same = same_cls & (a["n_cross"] == b["n_cross"]) & (a["n_cross"] > 0)
        idx = torch.nonzero(same).squeeze(1)
        k = (a["n_cross"][idx] - 1).long()
        ga = a["g"][k, idx]
        gb = b["g"][k, idx]
        dgs.append((gb - ga).abs() / ga.abs())
        maxc = a["r_hit"].shape[0] if "r_hit" in a else 0
        for c in range(maxc):
            m = same & (a["n_cross"] > c)
            if "r_hit" in b:
                errs["r_hit"].append(((b["r_hit"][c][m] - a["r_hit"][c][m]).abs() / a["r_hit"][c][m]))
            if "g" in b:
                errs["g"].append(((b["g"][c][m] - a["g"][c][m]).abs() / a["g"][c][m].abs()))
            if "phi_hit" in a and "phi_hit" in b:
                errs["phi_hit"].append(_wrap_abs(b["phi_hit"][c][m] - a["phi_hit"][c][m]))
        for f, m in (("flux", same), ("intensity", same_cls)):
            if f in a and f in b:
                peak = float(a[f].abs().max().item()) or 1.0
                errs[f].append((b[f][m] - a[f][m]).abs() / peak)
        esc = same_cls & (a["cls"] == 2)
        if "theta_inf" in a and "theta_inf" in b:
            errs["theta_inf"].append((b["theta_inf"][esc] - a["theta_inf"][esc]).abs())
        if "phi_inf" in a and "phi_inf" in b:
            errs["phi_inf"].append(_wrap_abs(b["phi_inf"][esc] - a["phi_inf"][esc]))
    dg = torch.cat(dgs)
    q = torch.quantile(dg[: 16_000_000].float(), torch.tensor([0.5, 0.999], device=dg.device)).tolist() \
        if dg.numel() else [None, None]
    units = {"r_hit": "relative", "g": "relative", "phi_hit": "rad (mod 2 pi)", "flux": "of the frame's peak",
             "intensity": "of the frame's peak", "theta_inf": "rad", "phi_inf": "rad (mod 2 pi)"}
    fields = {f: _stats(torch.cat(v), units[f]) for f, v in errs.items() if v}
    return {"class_agreement": agree / total, "dg_over_g_median": q[0], "dg_over_g_p999": q[1],
            "dg_over_g_max": float(dg.max().item()) if dg.numel() else None, "pixels_compared": int(dg.numel()),
            "fields": fields, "reference": reference}


def run_ours(args, rank: int, world: int, dist):
    import torch

    from blackhole_b200 import _abi, kerr

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    lib = _abi.load_library()
    wl = WORKLOADS[args.workload]
    integ = "dp45" if wl["integrator"] == 1 else "rk4"
    stream = torch.cuda.Stream(device=dev)

    precisions = [args.precision]
    if args.compare and args.precision != "fp64":
        precisions = ["fp64", args.precision]
    runs = {p: time_precision(args, p, dev, stream, dist) for p in precisions}
    head = runs[args.precision]
    rays_per_step = sum(s.width * s.height for s in head["scenes"])
    fm = head["frame_ms"]
    extra = {"launch_config": head["launch_cfg"],
             "frame_latency_ms": {"p50": float(np.percentile(fm, 50)), "p99": float(np.percentile(fm, 99)),
                                  "max": float(fm.max()), "frames": int(len(fm))}}
    value = rays_per_step * args.steps * world / (head["elapsed_ms"] * 1e-3)
    if "fp64" in runs and args.precision != "fp64":
        f = runs["fp64"]
        extra["fp64_plain"] = {"value": rays_per_step * args.steps * world / (f["elapsed_ms"] * 1e-3),
                               "unit": UNIT, "ms_per_step": f["elapsed_ms"] / args.steps,
                               "steps_per_render": f["total_steps"], "clocks": f["clocks"]}
        extra["speedup_vs_fp64_plain"] = value / extra["fp64_plain"]["value"]
        extra["accuracy_vs_fp64"] = accuracy(f["outs"], head["outs"])

    drift = {"definition": CARTER_DRIFT_DEF}
    for p, r in runs.items():
        s0 = r["scenes"][0]
        drift[p] = carter_drift_stats(lambda o, s0=s0: kerr.trace_image(s0, o, stream=stream),
                                      s0.width * s0.height, dev)
        drift[p]["frame"] = f"first frame of the workload ({s0.width}x{s0.height}, {p})"
    extra["carter_drift"] = drift

    # ---- end to end through the host-buffer C entry point (pinned host memory) ----
    e2e = None
    out_bytes = sum(t.numel() * t.element_size() for o in head["outs"] for t in o.values())
    if rank == 0 and out_bytes <= (4 << 30):  # pinned host copies of the outputs must stay modest
        scenes = head["scenes"]
        pinned = []
        for s in scenes:
            d = {}
            n_frame = s.width * s.height
            for fld in OUT_FIELDS_USED:
                shape = (s.max_crossings * n_frame,) if fld in _abi.PLANE_FIELDS else (n_frame,)
                dt = torch.int32 if fld in _abi.INT_FIELDS else torch.float64
                d[fld] = torch.empty(shape, dtype=dt).pin_memory()
            pinned.append(d)
        structs = []
        for d in pinned:
            o = _abi.KerrImageOut()
            for fld, t in d.items():
                setattr(o, fld, t.data_ptr())
            structs.append(o)
        d2h = sum(t.numel() * t.element_size() for d in pinned for t in d.values())
        h2d = C.sizeof(_abi.KerrScene) * len(scenes)
        for s, o in zip(scenes, structs):  # warm the host path's cached buffers
            _abi.check(lib.bh_kerr_trace_image_host(C.byref(s), C.byref(o)))
        e2e_steps = max(1, min(args.steps, 3))
        w0 = time.perf_counter()
        for _ in range(e2e_steps):
            for s, o in zip(scenes, structs):
                _abi.check(lib.bh_kerr_trace_image_host(C.byref(s), C.byref(o)))
        w1 = time.perf_counter()
        e2e = {"value": rays_per_step * e2e_steps / (w1 - w0), "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "api": "bh_kerr_trace_image_host"}

    # ---- roofline of the headline tracing kernel ----
    fp64 = args.precision == "fp64"
    peak = C.c_double(0.0)
    _check_probe(fma_probe().bh_bench_fma_peak(1 if fp64 else 0, 5, C.byref(peak)))
    mean_launch_s = statistics.mean(head["launch_ms"]) * 1e-3
    flops_per_launch = FLOPS_PER_STEP[integ] * head["total_steps"]
    achieved = flops_per_launch / mean_launch_s / 1e12
    kname = "k_trace_batch_fp64" if fp64 else "k_trace_batch_mixed"
    roofline = {"bound": "fp64" if fp64 else "fp32", "achieved": achieved, "peak": peak.value,
                "unit": "TFLOP/s", "frac": achieved / peak.value if peak.value else None, "traffic": None,
                "peak_source": "this repository's own FMA-pipe probe (bh_bench_fma_peak, lib/libbh_bench_probe.so; MEASURED_PEAKS.json has no FP32/FP64 figure), FMA = 2 FLOPs",
                "flops_per_step": FLOPS_PER_STEP[integ], "steps_per_launch": head["total_steps"],
                "kernel": f"{kname}<{1 if integ == 'dp45' else 0}>",
                "launch_ms_mean": statistics.mean(head["launch_ms"]),
                "launch_ms_min": min(head["launch_ms"]), "launch_ms_max": max(head["launch_ms"])}
    return dict(value=value, ms_per_step=head["elapsed_ms"] / args.steps, e2e=e2e, roofline=roofline,
                clocks=head["clocks"], total_steps=head["total_steps"], rays_per_step=rays_per_step,
                launches=len(runs) * args.steps, extra=extra)



def _timed_launches(fn, stream, steps: int, warmup: int):
    """CUDA-event times (ms) of ``steps`` calls of fn on ``stream`` after ``warmup``."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        out.append((a, b))
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in out]


LEGACY_SCENE = ("2048x2048 Blender-bridge camera (bridge defaults, fov 1.0, 600 steps of 0.08), a = 0.9, "
                "camera at 10 rs and 60 deg from the spin axis, disk and background on")


def time_legacy_launch(launch, steps: int = 5, warmup: int = 2) -> dict:
    """Frames of the reference's render launch ABI, bh_launch_geodesic_kernel,
    on one bridge-camera scene (device framebuffer, CUDA events on the
    launching stream, which is the legacy default stream for both
    implementations here)."""
    import torch

    from blackhole_b200 import legacy

    p = legacy.bridge_params(0.9, 10.0, math.radians(60.0), 1.0, 2048, 2048)
    fb = torch.empty(p.width * p.height * 4, dtype=torch.float32, device="cuda")
    ts = _timed_launches(lambda: launch(p, fb), torch.cuda.current_stream(), steps, warmup)
    ms = statistics.median(ts)
    return {"value": p.width * p.height / (ms * 1e-3), "unit": UNIT, "ms_per_frame": ms, "frames": steps,
            "scene": LEGACY_SCENE, "api": "bh_launch_geodesic_kernel"}


def run_surrogate(args, rank: int, world: int, dist):
    """The learned-surrogate workload: one step = one bh_surrogate_trace_image
    render of the 2048^2 a = 0.9 disk frame."""
    import torch

    from blackhole_b200 import _abi, kerr
    from blackhole_b200 import surrogate as S

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    lib = _abi.load_library()
    if not SURROGATE_WEIGHTS.exists():
        raise RuntimeError(f"{SURROGATE_WEIGHTS} missing: python -m blackhole_b200.train_surrogate")
    net = S.Surrogate(max_batch=128)
    net.load(SURROGATE_WEIGHTS)
    stream = torch.cuda.Stream(device=dev)
    smx = scenes_for(args.workload, 1)[0]
    s64 = scenes_for(args.workload, 0)[0]
    n = smx.width * smx.height
    outs = kerr.alloc_image_outputs(smx, device=dev, fields=list(OUT_FIELDS_USED))

    def render():
        net.trace_image(smx, outs, stream=stream)

    sampler = ClockSampler(dev.index if "CUDA_VISIBLE_DEVICES" not in os.environ else 0)
    sampler.start()
    sampler.wait_first_sample()
    for _ in range(args.warmup):
        render()
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    sampler.lines.clear()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t0.record(stream)
    for a, b in steps_ev:
        a.record(stream)
        render()
        b.record(stream)
    t1.record(stream)
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    if dist is not None:
        dist.barrier()
    elapsed_ms = t0.elapsed_time(t1)
    if dist is not None:
        t = torch.tensor([elapsed_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    render_ms = [a.elapsed_time(b) for a, b in steps_ev]
    stats = net.last_stats()
    value = n * args.steps * world / (elapsed_ms * 1e-3)

    # ---- the plain integrators on the same scene (same run, same box) ----
    o64 = kerr.alloc_image_outputs(s64, device=dev, fields=list(OUT_FIELDS_USED))
    omx = kerr.alloc_image_outputs(smx, device=dev, fields=list(OUT_FIELDS_USED))
    ms64 = _timed_launches(lambda: kerr.trace_image(s64, o64, stream=stream), stream, 2, 1)
    msmx = _timed_launches(lambda: kerr.trace_image(smx, omx, stream=stream), stream, 2, 1)
    from blackhole_b200._abi import default_scene

    c0 = default_scene(width=256, height=256, spin=0.9, theta_obs=math.radians(60.0), integrator=0,
                       max_crossings=1, precision=0)
    oc0 = kerr.alloc_image_outputs(c0, device=dev, fields=["cls", "steps"])
    msc0 = _timed_launches(lambda: kerr.trace_image(c0, oc0, stream=stream), stream, 2, 1)
    fp64_dp45 = n / (statistics.mean(ms64) * 1e-3)
    fp64_rk4 = 256 * 256 / (statistics.mean(msc0) * 1e-3)
    # ---- the closed-form tracer (BH_INTEGRATOR_ANALYTIC) on the same frame, FP64 ----
    san = _abi.KerrScene.from_buffer_copy(s64)
    san.integrator = _abi.INTEGRATOR_ANALYTIC
    oan = kerr.alloc_image_outputs(san, device=dev, fields=list(OUT_FIELDS_USED))
    ms_an = _timed_launches(lambda: kerr.trace_image(san, oan, stream=stream), stream, 3, 1)
    disk_fields = [f for f in OUT_FIELDS_USED if f not in ("phi_hit", "phi_inf")]
    oan_d = kerr.alloc_image_outputs(san, device=dev, fields=disk_fields)
    ms_an_d = _timed_launches(lambda: kerr.trace_image(san, oan_d, stream=stream), stream, 3, 1)
    # ---- ablation at equal outputs: the same render asked for the disk fields only ----
    outs_d = kerr.alloc_image_outputs(smx, device=dev, fields=disk_fields)
    ms_sd = _timed_launches(lambda: net.trace_image(smx, outs_d, stream=stream), stream, 3, 1)
    steps64 = int(o64["steps"].sum().item())
    extra = {
        "fp64_plain": {"value": fp64_dp45, "unit": UNIT, "ms_per_step": statistics.mean(ms64),
                       "method": f"FP64 DP45 rtol 1e-8 on the same {smx.width}x{smx.height} frame",
                       "steps_per_ray": steps64 / n},
        "fp64_plain_rk4": {"value": fp64_rk4, "unit": UNIT, "ms_per_step": statistics.mean(msc0),
                           "method": "FP64 RK4 h = 0.02 min(r, 20), the plain method of the 256^2 frame of this "
                                     "scene (rays/s measured on that frame)",
                           "steps_per_ray": float(oc0["steps"].double().mean().item())},
        "mixed_integrator": {"value": n / (statistics.mean(msmx) * 1e-3), "unit": UNIT,
                             "ms_per_step": statistics.mean(msmx), "method": "mixed-precision DP45, every pixel"},
        "speedup_vs_fp64_plain": value / fp64_dp45,
        "speedup_vs_fp64_rk4": value / fp64_rk4,
        "surrogate_stats": stats,
        "accuracy_vs_fp64": accuracy([o64], [outs]),
        "accuracy_vs_closed_form": accuracy(
            [oan], [outs], reference="this run's closed-form FP64 tracer: exact at the escape radius, where the "
                                     "DP45 stepper reports escape angles after its last step's overshoot"),
        "render_ms": {"mean": statistics.mean(render_ms), "min": min(render_ms), "max": max(render_ms)},
        "steps_per_s_note": "FP64 DP45 accepted steps of the same frame per second of render: the integration "
                            "the render stands in for (its own integrator steps, on rejected pixels: "
                            f"{int(outs['steps'].sum().item())} per render)",
    }
    extra["analytic"] = {
        "value": n / (statistics.mean(ms_an) * 1e-3), "unit": UNIT, "ms_per_step": statistics.mean(ms_an),
        "method": "every ray in closed form in Mino time (Jacobi sn/cn, Carlson R_J, Bulirsch cel), FP64, "
                  "all outputs incl. azimuths; DP45 on the rays it does not cover",
        "speedup_vs_fp64_plain": statistics.mean(ms64) / statistics.mean(ms_an),
        "stepped_pixels": int((oan["steps"] > 0).sum().item()),
        "accuracy_vs_fp64": accuracy([o64], [oan]),
        "disk_outputs_only": {"value": n / (statistics.mean(ms_an_d) * 1e-3), "unit": UNIT,
                              "ms_per_step": statistics.mean(ms_an_d), "fields": disk_fields,
                              "speedup_vs_fp64_plain": statistics.mean(ms64) / statistics.mean(ms_an_d)},
    }
    extra["carter_drift"] = {
        "definition": CARTER_DRIFT_DEF,
        "surrogate_render": carter_drift_stats(lambda o: net.trace_image(smx, o, stream=stream), n, dev),
        "fp64_dp45": carter_drift_stats(lambda o: kerr.trace_image(s64, o, stream=stream), n, dev),
        "mixed_dp45": carter_drift_stats(lambda o: kerr.trace_image(smx, o, stream=stream), n, dev),
    }
    extra["ablation_equal_outputs"] = {
        "all_fields": {"fields": list(OUT_FIELDS_USED), "surrogate_ms": statistics.mean(render_ms),
                       "closed_form_ms": statistics.mean(ms_an), "mixed_dp45_ms": statistics.mean(msmx)},
        "disk_fields": {"fields": disk_fields, "surrogate_ms": statistics.mean(ms_sd),
                        "closed_form_ms": statistics.mean(ms_an_d)},
        "note": "the renderer without a trained network sends every pixel to its fallback, the closed-form "
                "tracer; both renders give every field from an exact solve (accuracy keys above)",
    }

    # ---- network inference alone: the tensor-core kernel's roofline ----
    inp = S.grid_inputs(smx, device=dev, stream=stream)
    head = torch.empty(n, 16, dtype=torch.float32, device=dev)
    fwd_ms = _timed_launches(lambda: net.forward(inp, head, stream=stream), stream, 5, 2)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("bf16_tflops")
    achieved = SURROGATE_FLOPS_PER_RAY * n / (statistics.mean(fwd_ms) * 1e-3) / 1e12
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak or 1590.0, "unit": "TFLOP/s",
                "frac": achieved / (peak or 1590.0),
                "traffic": INFER_DRAM_BYTES_2048 if (smx.width, smx.height) == (2048, 2048) else None,
                "traffic_unit": "bytes per launch (dram read + write, ncu)",
                "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst, of measured)" if peak else "fallback 1.59 PF",
                "kernel": "k_mlp_infer", "flops_per_ray": SURROGATE_FLOPS_PER_RAY,
                "mma_flops_per_ray_executed": SURROGATE_MMA_FLOPS_PER_RAY, "rays_per_launch": n,
                "launch_ms_mean": statistics.mean(fwd_ms),
                "note": "network inference timed alone on the frame's inputs; a render also runs the refinement "
                        "kernel (FP64 set-up, FP32 quadrature) concurrently and the integrator on rejected pixels"}
    extra["stage_ms"] = {"network_inference": statistics.mean(fwd_ms),
                         "render_total": statistics.mean(render_ms)}

    # ---- end to end through the host-buffer C entry point (pinned host memory) ----
    e2e = None
    if rank == 0:
        fields = OUT_FIELDS_USED  # the headline render's outputs, all copied back
        pinned = {f: torch.empty(n * (smx.max_crossings if f in _abi.PLANE_FIELDS else 1),
                                 dtype=torch.int32 if f in _abi.INT_FIELDS else torch.float64).pin_memory()
                  for f in fields}
        o = _abi.KerrImageOut()
        for f, t in pinned.items():
            setattr(o, f, t.data_ptr())
        pol = _abi.SurrogatePolicy(0.99, 1, 0.05, 0, 0)
        _abi.check(lib.bh_surrogate_trace_image_host(net._h, C.byref(smx), C.byref(o), C.byref(pol)))
        k = max(1, min(args.steps, 3))
        w0 = time.perf_counter()
        for _ in range(k):
            _abi.check(lib.bh_surrogate_trace_image_host(net._h, C.byref(smx), C.byref(o), C.byref(pol)))
        w1 = time.perf_counter()
        e2e = {"value": n * k / (w1 - w0), "unit": UNIT, "h2d_bytes_per_step": C.sizeof(_abi.KerrScene),
               "d2h_bytes_per_step": sum(t.numel() * t.element_size() for t in pinned.values()),
               "api": "bh_surrogate_trace_image_host", "fields": list(fields)}
    chunks = 2  # the renderer's default chunk count (BH_SurrogatePolicy.chunks = 0)
    # inputs, chunks x (inference, refinement), the closed-form and DP45 fallback tracers
    launches = (1 + 2 * chunks + 2) * args.steps
    return dict(value=value, ms_per_step=elapsed_ms / args.steps, e2e=e2e, roofline=roofline, clocks=clocks,
                total_steps=steps64, rays_per_step=n, launches=launches, extra=extra)


def run_analytic(args, rank: int, world: int, dist):
    """The closed-form tracer: one step = one bh_kerr_trace_image of the frame
    with integrator BH_INTEGRATOR_ANALYTIC (FP64; DP45 on the rays it does
    not cover), the bench line's output fields; the FP64 DP45 tracer on the
    same frame is timed beside it and is the accuracy reference."""
    import torch

    from blackhole_b200 import _abi, kerr

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    lib = _abi.load_library()
    stream = torch.cuda.Stream(device=dev)
    s = scenes_for(args.workload, 0)[0]
    n = s.width * s.height
    outs = kerr.alloc_image_outputs(s, device=dev, fields=list(OUT_FIELDS_USED))

    def render():
        kerr.trace_image(s, outs, stream=stream)

    sampler = ClockSampler(dev.index if "CUDA_VISIBLE_DEVICES" not in os.environ else 0)
    sampler.start()
    sampler.wait_first_sample()
    for _ in range(args.warmup):
        render()
    torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    sampler.lines.clear()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        render()
    t1.record(stream)
    torch.cuda.synchronize(dev)
    clocks = sampler.stop()
    if dist is not None:
        dist.barrier()
    elapsed_ms = t0.elapsed_time(t1)
    if dist is not None:
        t = torch.tensor([elapsed_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    ms = elapsed_ms / args.steps
    value = n * args.steps * world / (elapsed_ms * 1e-3)

    s64 = _abi.KerrScene.from_buffer_copy(s)
    s64.integrator = _abi.INTEGRATOR_DP45
    o64 = kerr.alloc_image_outputs(s64, device=dev, fields=list(OUT_FIELDS_USED))
    ms64 = statistics.mean(_timed_launches(lambda: kerr.trace_image(s64, o64, stream=stream), stream, 2, 1))
    disk_fields = [f for f in OUT_FIELDS_USED if f not in ("phi_hit", "phi_inf")]
    od = kerr.alloc_image_outputs(s, device=dev, fields=disk_fields)
    ms_d = statistics.mean(_timed_launches(lambda: kerr.trace_image(s, od, stream=stream), stream, 5, 2))
    extra = {
        "fp64_plain": {"value": n / (ms64 * 1e-3), "unit": UNIT, "ms_per_step": ms64,
                       "method": f"FP64 DP45 rtol 1e-8 on the same {s.width}x{s.height} frame"},
        "speedup_vs_fp64_plain": ms64 / ms,
        "accuracy_vs_fp64": accuracy([o64], [outs]),
        "stepped_pixels": int((outs["steps"] > 0).sum().item()),
        "disk_outputs_only": {"value": n / (ms_d * 1e-3), "unit": UNIT, "ms_per_step": ms_d, "fields": disk_fields,
                              "speedup_vs_fp64_plain": ms64 / ms_d},
    }
    # Outputs are the only HBM traffic (no inputs): the roofline below is the
    # HBM one, far from binding; the kernel is bound by instruction fetch
    # (profiles/k_trace_image_analytic_disk1_512.md).
    out_bytes = sum(t.numel() * t.element_size() for t in outs.values())
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs")
    achieved = out_bytes / (ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak or 6650.0, "unit": "GB/s",
                "frac": achieved / (peak or 6650.0), "traffic": None, "kernel": "k_trace_image_analytic",
                "bytes_per_launch": out_bytes,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peak else "fallback 6.65 TB/s",
                "note": "algorithmic bytes = the outputs written; the kernel is bound by instruction fetch, not HBM"}
    e2e = None
    if rank == 0:
        fields = ("cls", "n_cross", "r_hit", "g", "flux", "intensity")
        pinned = {f: torch.empty(n * (s.max_crossings if f in _abi.PLANE_FIELDS else 1),
                                 dtype=torch.int32 if f in _abi.INT_FIELDS else torch.float64).pin_memory()
                  for f in fields}
        o = _abi.KerrImageOut()
        for f, t in pinned.items():
            setattr(o, f, t.data_ptr())
        _abi.check(lib.bh_kerr_trace_image_host(C.byref(s), C.byref(o)))
        k = max(1, min(args.steps, 3))
        w0 = time.perf_counter()
        for _ in range(k):
            _abi.check(lib.bh_kerr_trace_image_host(C.byref(s), C.byref(o)))
        w1 = time.perf_counter()
        e2e = {"value": n * k / (w1 - w0), "unit": UNIT, "h2d_bytes_per_step": C.sizeof(_abi.KerrScene),
               "d2h_bytes_per_step": sum(t.numel() * t.element_size() for t in pinned.values()),
               "api": "bh_kerr_trace_image_host", "fields": list(fields)}
    # per step: the closed-form kernel and the DP45 list tracer on what it leaves
    return dict(value=value, ms_per_step=ms, e2e=e2e, roofline=roofline, clocks=clocks,
                total_steps=int(outs["steps"].sum().item()), rays_per_step=n, launches=2 * args.steps, extra=extra)


def run_rt(args, rank: int, world: int, dist):
    """The volumetric workload: one step = one render of I_nu through the
    synthetic 128 x 64 x 64 torus (DP45 rays, <= 2000 steps), at the
    requested precision; the FP64 render of the same frame is timed beside it
    and is the accuracy reference."""
    import torch

    from blackhole_b200 import kerr
    from blackhole_b200 import rt

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    med = rt.Medium(device=dev)
    lut = rt.Lut(device=dev)
    prm = rt.rt_defaults()
    wl = WORKLOADS[args.workload]
    prec = 1 if args.precision == "mixed" else 0

    def scene(pr):
        return kerr.scene(width=wl["width"], height=wl["height"], spin=0.94, theta_obs=math.radians(17.0),
                          integrator=1, precision=pr, max_crossings=1, max_steps=2000, alpha_min=-20, alpha_max=20,
                          beta_min=-20, beta_max=20)

    s = scene(prec)
    n = s.width * s.height
    outs = None

    def render():
        nonlocal outs
        outs = rt.trace(s, med, lut, prm, outs=outs, stream=stream)

    sampler = ClockSampler(dev.index if "CUDA_VISIBLE_DEVICES" not in os.environ else 0)
    sampler.start()
    sampler.wait_first_sample()
    ms = _timed_launches(render, stream, args.steps, args.warmup)
    clocks = sampler.stop()
    elapsed_ms = sum(ms)
    if dist is not None:
        t = torch.tensor([elapsed_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
    value = n * args.steps * world / (elapsed_ms * 1e-3)
    steps = int(outs["steps"].sum().item())
    cls = outs["cls"].cpu().numpy()
    extra = {"rt": {"steps_per_ray": steps / n, "classes": {str(c): int((cls == c).sum()) for c in np.unique(cls)},
                    "lit_fraction": float((outs["i_nu"] > 0).double().mean().item()),
                    "tau_median": float(outs["tau"].median().item()), "nu_hz": prm.nu_hz,
                    "ds_max_M": prm.ds_max}}
    if prec == 1:
        s64 = scene(0)
        o64 = None

        def render64():
            nonlocal o64
            o64 = rt.trace(s64, med, lut, prm, outs=o64, stream=stream)

        ms64 = _timed_launches(render64, stream, 2, 1)
        a, b = outs, o64
        lit = (b["i_nu"] > 1e-6 * b["i_nu"].max()) & (a["cls"] == b["cls"])
        rel = ((a["i_nu"][lit] - b["i_nu"][lit]).abs() / b["i_nu"][lit]).float()
        q = torch.quantile(rel, torch.tensor([0.5, 0.99], device=rel.device)).tolist()
        extra["fp64_plain"] = {"value": n / (statistics.mean(ms64) * 1e-3), "unit": UNIT,
                               "ms_per_step": statistics.mean(ms64), "method": "FP64 DP45 transfer, same frame"}
        extra["speedup_vs_fp64_plain"] = value / extra["fp64_plain"]["value"]
        extra["accuracy_vs_fp64"] = {"class_agreement": float((a["cls"] == b["cls"]).double().mean().item()),
                                     "i_nu_rel_median": q[0], "i_nu_rel_p99": q[1],
                                     "pixels_compared": int(lit.sum().item()),
                                     "note": "the mixed steps differ, so samples sit elsewhere on each ray: "
                                             "differences are at the sampling's discretization level"}
    from blackhole_b200 import _abi

    peak = C.c_double(0.0)
    _check_probe(fma_probe().bh_bench_fma_peak(1 if prec == 0 else 0, 5, C.byref(peak)))
    achieved = FLOPS_PER_STEP["rt"] * steps / (statistics.mean(ms) * 1e-3) / 1e12
    roofline = {"bound": "fp64" if prec == 0 else "fp32", "achieved": achieved, "peak": peak.value,
                "unit": "TFLOP/s", "frac": achieved / peak.value if peak.value else None, "traffic": None,
                "peak_source": "this repository's own FMA-pipe probe (bh_bench_fma_peak, lib/libbh_bench_probe.so; MEASURED_PEAKS.json has no FP32/FP64 figure), FMA = 2 FLOPs",
                "flops_per_step": FLOPS_PER_STEP["rt"], "steps_per_launch": steps,
                "kernel": "k_trace_rt_fp64" if prec == 0 else "k_trace_rt_mixed",
                "launch_ms_mean": statistics.mean(ms),
                "note": "DP45 geodesic step plus its medium samples; the grid and table are L2-resident"}
    # ---- end to end: medium and table uploaded from pinned host memory, I_nu and tau read back ----
    e2e = None
    if rank == 0:
        cells_h = med.cells.cpu().pin_memory()
        lut_h = lut.table.cpu().pin_memory()
        out_h = {k: torch.empty(n, dtype=torch.float64).pin_memory() for k in ("i_nu", "tau")}

        def step_e2e():
            med.cells.copy_(cells_h, non_blocking=True)
            lut.table.copy_(lut_h, non_blocking=True)
            torch.cuda.current_stream().synchronize()
            o = rt.trace(s, med, lut, prm)
            for k in out_h:
                out_h[k].copy_(o[k], non_blocking=True)
            torch.cuda.synchronize()

        step_e2e()
        k = max(1, min(args.steps, 3))
        w0 = time.perf_counter()
        for _ in range(k):
            step_e2e()
        w1 = time.perf_counter()
        e2e = {"value": n * k / (w1 - w0), "unit": UNIT,
               "h2d_bytes_per_step": cells_h.numel() * cells_h.element_size() + lut_h.numel() * lut_h.element_size(),
               "d2h_bytes_per_step": sum(t.numel() * t.element_size() for t in out_h.values()),
               "api": "bh_kerr_trace_rt (device buffers) with the medium uploaded and I_nu, tau read back"}
    d = lut.desc
    cpu_inputs = {"scene": scene(0), "cells": med.cells.cpu().numpy(), "lut": lut.table.cpu().numpy(),
                  "log_theta": (d.log_theta_min, d.log_theta_max), "log_x": (d.log_x_min, d.log_x_max), "rt": prm}
    return dict(value=value, ms_per_step=elapsed_ms / args.steps, e2e=e2e, roofline=roofline, clocks=clocks,
                total_steps=steps, rays_per_step=n, launches=args.steps, extra=extra, cpu_inputs=cpu_inputs)

# ---------------------------------------------------------------------------
# reference arm: the reference's compiled CPU code on the host cores
# ---------------------------------------------------------------------------
def cpu_reference(workload: str, budget_s: float, seed: int = 7):
    """Time oracle/_ref (reference-compiled potentials) on a bounded random
    sample of the workload's pixels until ~budget_s of wall time is spent."""
    from oracle.pyoracle import RefLib, default_threads

    lib = RefLib()
    threads = default_threads()
    scenes = scenes_for(workload, 0)
    for s in scenes:  # the reference's CPU path steps every ray (DP45 for the closed-form workloads)
        if s.integrator == 2:
            s.integrator = 1
    n_frame = scenes[0].width * scenes[0].height
    rng = np.random.default_rng(seed)
    done = 0
    chunk = max(64, 4 * threads)
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < budget_s:
        for s in scenes:
            pix = rng.integers(0, n_frame, chunk)
            lib.trace_pixels(s, pix, threads=threads)
            done += chunk
    el = time.perf_counter() - t0
    return {"value": done / el, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{done} random pixels spread over the {len(scenes)} frames of {workload}, "
                      f"{el:.1f} s wall on {threads} threads (oracle/_ref: reference kerrPotentials)"}


def reference_gpu_kernel() -> dict:
    """The reference's own FP32 render kernel (geodesicTraceFp32, variant 0 of
    its bh_launch_geodesic_kernel; oracle/_ref/libbh_ref_render.so, compiled
    from its source for sm_100a) on the bridge-camera scene, for context: FP32
    fixed-step stepping and art-directed shading, not this metric's method."""
    lib_path = ROOT / "oracle" / "_ref" / "libbh_ref_render.so"
    try:
        import torch

        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
        if not lib_path.exists():
            return {"unavailable": "oracle/_ref/libbh_ref_render.so not built (reference sources absent at build)"}
        from blackhole_b200 import legacy

        ref = C.CDLL(str(lib_path))
        ref.bh_launch_geodesic_kernel.argtypes = [C.c_void_p, C.POINTER(legacy.LaunchParams), C.c_int, C.c_void_p]
        ref.bh_launch_geodesic_kernel.restype = C.c_int

        def launch(p, fb):
            if ref.bh_launch_geodesic_kernel(C.c_void_p(fb.data_ptr()), C.byref(p), 0, None) != 0:
                raise RuntimeError("reference bh_launch_geodesic_kernel failed")

        out = time_legacy_launch(launch)
        out["kernel"] = "geodesicTraceFp32 (reference build, FP32)"
        return out
    except Exception as e:  # context only: never fail the reference line over it
        return {"unavailable": f"{type(e).__name__}: {e}"}


def cpu_reference_rt(inp: dict, budget_s: float, seed: int = 7):
    """Time the CPU restatement of the transfer (oracle rt_oracle.hpp: FP64
    DP45 ray, the reference's synchrotron / Planck / rteStep physics) on a
    bounded random sample of the frame's pixels, all host threads."""
    from oracle.pyoracle import Oracle, default_threads

    o = Oracle()
    threads = default_threads()
    s = inp["scene"]
    n = s.width * s.height
    rng = np.random.default_rng(seed)
    done = 0
    chunk = max(32, 2 * threads)
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < budget_s:
        pix = rng.integers(0, n, chunk)
        p = inp["rt"]
        o.trace_rt(s, inp["cells"], (2.0, 50.0), inp["lut"], inp["log_theta"], inp["log_x"], p.nu_hz, p.length_cm,
                   p.ds_max, p.min_transmit, pix=pix, threads=threads)
        done += chunk
    el = time.perf_counter() - t0
    return {"value": done / el, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{done} random pixels of the {s.width}x{s.height} transfer frame, {el:.1f} s wall on "
                      f"{threads} threads (oracle: FP64 restatement of the transfer)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", choices=tuple(WORKLOADS), default="c4_2048")
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="mixed")
    ap.add_argument("--compare", action=argparse.BooleanOptionalAction, default=True,
                    help="also time the FP64 plain path and report the accuracy against it")
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of CPU baseline sampling")
    ap.add_argument("--autotune", action=argparse.BooleanOptionalAction, default=True,
                    help="autotune the persistent-grid shape before timing")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", 1))
    rank = int(os.environ.get("RANK", 0))
    wl = WORKLOADS[args.workload]
    if "generator" in wl:
        config = {"workload": args.workload, "frames": 4096, "sizes": [64, 128, 256, 512], "spin": [0, 0.998],
                  "theta_obs_deg": [5, 89], "r_obs": "logU[100, 5000]", "seed": "per frame",
                  "integrator": "dp45" if wl["integrator"] == 1 else "rk4", "rtol": 1e-8, "atol": 1e-10,
                  "max_crossings": wl["max_crossings"], "image_plane_M": [-12, 12]}
    else:
        config = {"workload": args.workload, "frames": len(wl["frames"]), "width": wl["width"], "height": wl["height"],
                  "integrator": {0: "rk4", 1: "dp45", 2: "analytic"}[wl["integrator"]], "rtol": 1e-8, "atol": 1e-10,
                  "max_crossings": wl["max_crossings"], "r_obs": 1000.0, "image_plane_M": [-12, 12]}
    config.update({"parallelism": f"replicas{world}", "launch": "one persistent launch per step (CUDA graph)",
                   "l2": "no inputs; outputs written once per step, larger than L2"})
    if wl.get("sky"):
        config["sky"] = {"cubemap": f"6x{SKY_SIZE}x{SKY_SIZE} FP16", "stars": SKY_STARS, "seed": SKY_SEED,
                         "lookup": "nearest texel at the escape direction, added to the intensity"}
    if wl.get("rt"):
        config.update({"spin": 0.94, "theta_obs_deg": 17.0, "image_plane_M": [-20, 20], "max_steps": 2000,
                       "medium": "128x64x64 (log r 2..50 M, theta, phi) FP32 grid: Gaussian torus r_in 6, r_peak 12 "
                                 "x exp(GRF sigma 0.5, correlation 2 M)",
                       "emission": "thermal synchrotron, 256x256 FP32 table over (log Theta_e, log nu/nu_s), "
                                   "Kirchhoff absorption", "precision": args.precision,
                       "launch": "one persistent launch per step"})
    if wl.get("surrogate"):
        config.update({"spin": 0.9, "theta_obs_deg": 60.0, "method": "mixed precision + learned surrogate",
                       "network": "192 features -> 4 x 256 SiLU -> 16, BF16 weights, FP32 accumulation",
                       "weights": "blackhole_b200/data/surrogate_c4.npz (trained on 2^26 integrator rays)",
                       "policy": {"min_confidence": 0.99, "critical_band_M": 0.05, "verify": "radial kind"},
                       "launch": "7 launches per render on two streams: inputs, 2 x (inference, refinement), "
                                 "the closed-form tracer and DP45 on the rejected pixels",
                       "l2": f"outputs ({wl['width']}^2 pixels x 10 fields) written once per step, larger than L2"})

    if args.impl == "reference":
        if rank != 0:
            return
        cb = cpu_reference(args.workload, args.cpu_budget)
        line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config, "impl": "reference",
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        if args.workload == "c4_2048":
            line["gpu_kernel_context"] = reference_gpu_kernel()
        print(json.dumps(line))
        return

    dist = None
    if world > 1:
        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        dist = dist_mod
    if wl.get("analytic"):
        config.update({"spin": wl["frames"][0][0], "theta_obs_deg": wl["frames"][0][1], "precision": "fp64",
                       "method": "closed form in Mino time (BH_INTEGRATOR_ANALYTIC)",
                       "launch": "2 launches per step: the closed-form kernel, DP45 on the rays it does not cover"})
    if wl.get("surrogate"):
        res = run_surrogate(args, rank, world, dist)
    elif wl.get("analytic"):
        res = run_analytic(args, rank, world, dist)
    elif wl.get("rt"):
        res = run_rt(args, rank, world, dist)
    else:
        res = run_ours(args, rank, world, dist)
    if rank == 0:
        if world == 1 and args.workload == "c4_2048":
            from blackhole_b200 import legacy

            lr = time_legacy_launch(lambda p, fb: legacy.launch(p, fb, -1))
            lr["kernel"] = "k_trace_camera_mixed + shading (mixed DP45)"
            res["extra"]["legacy_render"] = lr
        cb = None
        if world == 1 and args.cpu_budget > 0:
            cb = cpu_reference_rt(res["cpu_inputs"], args.cpu_budget) if wl.get("rt") else \
                cpu_reference(args.workload, args.cpu_budget)
        line = {"metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": res["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "bf16+f32+f64" if wl.get("surrogate") else
                ("f64" if args.precision == "fp64" or wl.get("analytic") else "f32+f64"),
                "data": "synthetic", "config": config, "precision": "fp64" if wl.get("analytic") else args.precision,
                "steps_per_s": res["total_steps"] * args.steps * world / (res["ms_per_step"] * args.steps * 1e-3),
                **res["extra"],
                "e2e": res["e2e"], "roofline": res["roofline"], "cpu_baseline": cb, "clocks": res["clocks"],
                "gpu_launches": res["launches"]}
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
