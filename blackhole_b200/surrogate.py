"""Learned transfer function for Kerr image-plane rays (include/bh_surrogate.h).

A 4 x 256 SiLU MLP maps (alpha, beta, spin, cos theta_obs) -- through 134
features: the scaled inputs, the ray's constants of motion lambda and eta,
and 16 Fourier frequencies of each input -- to the ray's termination class,
its first two disk crossings, the redshift of the first and its escape
direction. Forward, backward and Adam run in the library's BF16 tensor-core
kernels with FP32 accumulation; training data are rays the library's own
integrator traced. Tensors are torch CUDA tensors (plumbing only).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _abi
from ._abi import AdamConfig, KerrImageOut, check

N_FEATURES = 192
N_FEATURES_USED = 134
HIDDEN = 256
HEAD = 16
LAYER_K = (192, 256, 256, 256, 256)
LAYER_N = (256, 256, 256, 256, 16)

# Head columns.
LOGITS = slice(0, 3)
COL_LNR1, COL_COSPHI1, COL_SINPHI1 = 3, 4, 5
COL_LNR2, COL_COSPHI2, COL_SINPHI2 = 6, 7, 8
COL_G1, COL_COSTH_INF, COL_COSPHI_INF, COL_SINPHI_INF = 9, 10, 11, 12


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _stream(stream) -> int | None:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


def param_count() -> int:
    return int(_abi.load_library().bh_surrogate_param_count())


def weight_slices() -> list[tuple[slice, slice]]:
    """(weight slice, bias slice) of each layer in the flat parameter vector."""
    out, off = [], 0
    for k, n in zip(LAYER_K, LAYER_N):
        out.append((slice(off, off + n * k), slice(off + n * k, off + n * k + n)))
        off += n * k + n
    return out


def features(inputs: torch.Tensor, stream=None) -> torch.Tensor:
    """BF16 features [n][192] of FP32 inputs [n][4]."""
    assert inputs.is_cuda and inputs.dtype == torch.float32 and inputs.shape[1] == 4
    inputs = inputs.contiguous()
    F = torch.empty(inputs.shape[0], N_FEATURES, dtype=torch.bfloat16, device=inputs.device)
    check(_abi.load_library().bh_surrogate_features(_ptr(inputs), inputs.shape[0], _ptr(F), _stream(stream)))
    return F


def bf16_gemm(A: torch.Tensor, B: torch.Tensor, stream=None) -> torch.Tensor:
    """C = A B^T (FP32) on the tensor cores for BF16 A [M][K], B [N][K]."""
    assert A.dtype == B.dtype == torch.bfloat16 and A.is_cuda and B.is_cuda
    A, B = A.contiguous(), B.contiguous()
    M, K = A.shape
    N = B.shape[0]
    assert B.shape[1] == K
    Cm = torch.empty(M, N, dtype=torch.float32, device=A.device)
    check(_abi.load_library().bh_bf16_gemm(_ptr(A), _ptr(B), M, N, K, _ptr(Cm), _stream(stream)))
    return Cm


def grid_inputs(scene, device="cuda", stream=None) -> torch.Tensor:
    """FP32 inputs [width*height][4] of a scene's pixel centres."""
    n = scene.width * scene.height
    inp = torch.empty(n, 4, dtype=torch.float32, device=device)
    check(_abi.load_library().bh_surrogate_grid_inputs(C.byref(scene), _ptr(inp), _stream(stream)))
    return inp


def make_targets(outs: dict, n: int, max_crossings: int, device="cuda", stream=None) -> torch.Tensor:
    """FP32 targets [n][16] from tracer output tensors (bh_kerr_trace_image layout)."""
    o = KerrImageOut()
    for k, v in outs.items():
        setattr(o, k, v.data_ptr())
    tg = torch.empty(n, 16, dtype=torch.float32, device=device)
    check(_abi.load_library().bh_surrogate_make_targets(C.byref(o), n, max_crossings, _ptr(tg), _stream(stream)))
    return tg


class Surrogate:
    """The network: FP32 master weights on the device, BF16 copies for the GEMMs."""

    def __init__(self, max_batch: int = 16384, seed: int = 0):
        lib = _abi.load_library()
        h = lib.bh_surrogate_create(max_batch, seed)
        if not h:
            raise RuntimeError(lib.bh_last_error().decode())
        self._h, self._lib = h, lib
        self.max_batch = max_batch
        self.n_params = param_count()

    def close(self):
        if getattr(self, "_h", None):
            self._lib.bh_surrogate_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self) -> np.ndarray:
        p = np.empty(self.n_params, np.float32)
        check(self._lib.bh_surrogate_get_params(self._h, p.ctypes.data, self.n_params))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        check(self._lib.bh_surrogate_set_params(self._h, p.ctypes.data, self.n_params))

    def get_state(self):
        """Adam moments (m, v) and step count."""
        m = np.empty(self.n_params, np.float32)
        v = np.empty(self.n_params, np.float32)
        step = C.c_int64(0)
        check(self._lib.bh_surrogate_get_state(self._h, m.ctypes.data, v.ctypes.data, self.n_params, C.byref(step)))
        return m, v, int(step.value)

    def set_state(self, m: np.ndarray, v: np.ndarray, step: int):
        m = np.ascontiguousarray(m, np.float32)
        v = np.ascontiguousarray(v, np.float32)
        check(self._lib.bh_surrogate_set_state(self._h, m.ctypes.data, v.ctypes.data, self.n_params, int(step)))

    def save(self, path, manifest: dict | None = None):
        """Checkpoint: parameters and Adam state in ``path`` (.npz), and beside
        it ``path`` + ``.json``, a manifest of what made it (``manifest``:
        seed, training and data configuration, optionally ``git_commit``;
        added here: the network's shapes, the SHA-256 of the parameters, the
        data configuration's hash, and the git commit of the source tree when
        the caller gave none and the tree is a git checkout)."""
        import hashlib
        import json
        import subprocess
        from pathlib import Path

        params = self.get_params()
        m, v, step = self.get_state()
        np.savez_compressed(path, params=params, adam_m=m, adam_v=v, adam_step=np.int64(step))
        man = dict(manifest or {})
        man.update({
            "format": "blackhole_b200 surrogate checkpoint 1",
            "param_count": int(self.n_params), "layer_k": list(LAYER_K), "layer_n": list(LAYER_N),
            "params_sha256": hashlib.sha256(params.tobytes()).hexdigest(), "adam_step": step,
        })
        if "data" in man:
            man["data_hash"] = hashlib.sha256(json.dumps(man["data"], sort_keys=True).encode()).hexdigest()
        if not man.get("git_commit"):  # the caller's, else the source tree's when it is a git checkout
            try:
                man["git_commit"] = subprocess.run(["git", "rev-parse", "HEAD"], capture_output=True, text=True,
                                                   cwd=Path(__file__).resolve().parent, check=True).stdout.strip()
            except (OSError, subprocess.CalledProcessError):
                man["git_commit"] = None
        Path(str(path) + ".json").write_text(json.dumps(man, indent=1, sort_keys=True) + "\n")

    def load(self, path):
        """Parameters, and the Adam state when the checkpoint carries it."""
        z = np.load(path)
        self.set_params(z["params"])
        if "adam_m" in z:
            self.set_state(z["adam_m"], z["adam_v"], int(z["adam_step"]))

    def forward(self, inputs: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        inputs = inputs.contiguous()
        n = inputs.shape[0]
        if out is None:
            out = torch.empty(n, HEAD, dtype=torch.float32, device=inputs.device)
        check(self._lib.bh_surrogate_forward(self._h, _ptr(inputs), n, _ptr(out), _stream(stream)))
        return out

    def gradients(self, inputs: torch.Tensor, targets: torch.Tensor, stream=None):
        grad = torch.empty(self.n_params, dtype=torch.float32, device=inputs.device)
        loss = torch.zeros(4, dtype=torch.float32, device=inputs.device)
        check(self._lib.bh_surrogate_gradients(self._h, _ptr(inputs.contiguous()), _ptr(targets.contiguous()),
                                               inputs.shape[0], _ptr(grad), _ptr(loss), _stream(stream)))
        return grad, loss

    def train_step(self, inputs: torch.Tensor, targets: torch.Tensor, lr: float, loss: torch.Tensor | None = None,
                   beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        cfg = AdamConfig(lr, beta1, beta2, eps)
        check(self._lib.bh_surrogate_train_step(self._h, _ptr(inputs), _ptr(targets), inputs.shape[0],
                                                C.byref(cfg), _ptr(loss), _stream(stream)))

    def trace_image(self, scene, outs: dict | None = None, min_confidence: float = 0.99, verify: int = 1,
                    critical_band: float = 0.05, refine_fp64: bool = False, chunks: int = 0, stream=None) -> dict:
        """Render a scene through the network with exact refinement and the
        integrator on rejected pixels (bh_surrogate_trace_image)."""
        from .kerr import _out_struct, alloc_image_outputs

        if outs is None:
            outs = alloc_image_outputs(scene)
        pol = _abi.SurrogatePolicy(min_confidence, verify, critical_band, int(refine_fp64), int(chunks))
        o = _out_struct(outs)
        check(self._lib.bh_surrogate_trace_image(self._h, C.byref(scene), C.byref(o), C.byref(pol),
                                                 _stream(stream)))
        return outs

    def trace_image_host(self, scene, fields=None, min_confidence: float = 0.99, verify: int = 1,
                         critical_band: float = 0.05, refine_fp64: bool = False, chunks: int = 0,
                         pinned: bool = True) -> dict:
        """The same render into host (numpy) buffers through
        bh_surrogate_trace_image_host; raises on -1 with the library's message.

        ``pinned``: the arrays are views of page-locked memory, so the library
        copies each chunk's rows while later chunks render; with False they
        are ordinary numpy arrays, copied after the render. The values are
        the same either way."""
        from .kerr import _out_struct, host_image_outputs

        if pinned:
            n = scene.width * scene.height
            mc = scene.max_crossings
            fields = fields or _abi.OUT_FIELDS
            ts = {k: torch.zeros((mc, n) if k in _abi.PLANE_FIELDS else (n,),
                                 dtype=torch.int32 if k in _abi.INT_FIELDS else torch.float64).pin_memory()
                  for k in fields}
            o = _out_struct(ts)
            arrs = {k: v.numpy() for k, v in ts.items()}  # views: each keeps its page-locked tensor alive
        else:
            arrs, o = host_image_outputs(scene, fields)
        pol = _abi.SurrogatePolicy(min_confidence, verify, critical_band, int(refine_fp64), int(chunks))
        check(self._lib.bh_surrogate_trace_image_host(self._h, C.byref(scene), C.byref(o), C.byref(pol)))
        return arrs

    def set_wait_limit(self, ns: int) -> None:
        """Limit of each bounded wait of the network's kernels (0: the default, 2 s)."""
        check(self._lib.bh_surrogate_set_wait_limit(self._h, int(ns)))

    def last_stats(self) -> dict:
        st = _abi.SurrogateStats()
        check(self._lib.bh_surrogate_last_stats(self._h, C.byref(st)))
        return {name: int(getattr(st, name)) for name, _ in st._fields_}

    def device_error(self) -> int:
        rc = self._lib.bh_surrogate_device_error(self._h)
        if rc < 0:
            check(rc)
        return rc


# ---- training data -------------------------------------------------------------


@dataclass
class RaySet:
    inputs: torch.Tensor   # [n][4] FP32
    targets: torch.Tensor  # [n][16] FP32


def training_scenes(n_frames: int, size: int, seed: int, window: float = 15.0, precision: int = 1):
    """Frames with a ~ U[0, 0.998], theta_obs ~ U[5, 89] deg and a random
    sub-pixel shift of the alpha, beta grid over [-window, window]: together
    the pixel centres cover the input domain uniformly."""
    from .kerr import scene

    out = []
    for f in range(n_frames):
        rng = np.random.default_rng([seed, f])
        a = float(rng.uniform(0.0, 0.998))
        th = math.radians(float(rng.uniform(5.0, 89.0)))
        d = 2.0 * window / size
        sa, sb = rng.uniform(-0.5, 0.5, 2) * d
        out.append(scene(width=size, height=size, spin=a, theta_obs=th, r_obs=1000.0,
                         alpha_min=-window + sa, alpha_max=window + sa, beta_min=-window + sb, beta_max=window + sb,
                         integrator=1, precision=precision, max_crossings=2))
    return out


def generate_rays(n_frames: int, size: int = 128, seed: int = 1, frames_per_batch: int = 256,
                  device="cuda") -> RaySet:
    """Trace n_frames random frames (DP45, mixed precision, two crossings)
    with the batched tracer and turn the outputs into training targets."""
    from .kerr import TraceBatch

    fields = ["cls", "n_cross", "r_hit", "phi_hit", "g", "theta_inf", "phi_inf"]
    n = n_frames * size * size
    inputs = torch.empty(n, 4, dtype=torch.float32, device=device)
    targets = torch.empty(n, 16, dtype=torch.float32, device=device)
    scenes = training_scenes(n_frames, size, seed)
    row = 0
    for f0 in range(0, n_frames, frames_per_batch):
        chunk = scenes[f0:f0 + frames_per_batch]
        b = TraceBatch(chunk, fields=fields)
        b.trace()
        for s, o in zip(chunk, b.outs):
            m = s.width * s.height
            inputs[row:row + m] = grid_inputs(s, device=device)
            targets[row:row + m] = make_targets(o, m, s.max_crossings, device=device)
            row += m
        torch.cuda.synchronize()
        b.close()
        del b
    return RaySet(inputs, targets)


def train(net: Surrogate, data: RaySet, epochs: float, batch: int = 16384, lr: float = 2e-3,
          lr_final: float = 5e-5, seed: int = 0, log_every: int = 0, log=print) -> list[dict]:
    """Adam with cosine learning-rate decay over shuffled mini-batches."""
    n = data.inputs.shape[0]
    steps_per_epoch = n // batch
    total = max(1, int(round(epochs * steps_per_epoch)))
    gen = torch.Generator(device=data.inputs.device)
    gen.manual_seed(seed)
    loss = torch.zeros(4, dtype=torch.float32, device=data.inputs.device)
    history = []
    perm = None
    for step in range(total):
        k = step % steps_per_epoch
        if k == 0:
            perm = torch.randperm(n, device=data.inputs.device, generator=gen)
        idx = perm[k * batch:(k + 1) * batch]
        x = data.inputs.index_select(0, idx)
        t = data.targets.index_select(0, idx)
        frac = step / max(1, total - 1)
        lr_s = lr_final + 0.5 * (lr - lr_final) * (1.0 + math.cos(math.pi * frac))
        net.train_step(x, t, lr_s, loss=loss)
        if log_every and (step % log_every == 0 or step == total - 1):
            v = loss.tolist()
            rec = {"step": step, "lr": lr_s, "ce": v[0] / max(v[3], 1), "reg": v[1] / batch,
                   "acc": v[2] / max(v[3], 1)}
            history.append(rec)
            if log:
                log(rec)
    return history
