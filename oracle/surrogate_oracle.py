"""CPU oracle of the learned transfer function (test infrastructure only).

A float64 numpy restatement of the network of include/bh_surrogate.h --
features, forward pass, loss, backward pass -- used by the tests to check the
GPU's tensor-core forward and backward kernels. The network has no
counterpart in the reference (its renderer integrates every pixel,
src/cuda/device_physics.cuh:912-1017); what is pinned here is the GPU
against this restatement, and the restatement against central finite
differences of its own loss.

``emulate=True`` rounds to BF16 at the points where the GPU stores BF16:
weights, features, hidden activations H, the loss gradient w.r.t. the head
and the back-propagated dY; everything else is exact float64 (the GPU
accumulates in FP32). ``emulate="f16"`` rounds the same points of the
forward pass to FP16 instead, as the fused inference kernel stores them
(training runs in BF16; inference evaluates the trained network in FP16).
"""
from __future__ import annotations

import numpy as np

LAYER_K = (192, 256, 256, 256, 256)
LAYER_N = (256, 256, 256, 256, 16)
FREQ = np.array([2.0 ** (k / 3.0) for k in range(16)], np.float32)


def bf16(x) -> np.ndarray:
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def f16(x) -> np.ndarray:
    """Round to the nearest FP16 (ties to even), returned as float64."""
    return np.asarray(x, np.float64).astype(np.float16).astype(np.float64)


def features(inputs: np.ndarray) -> np.ndarray:
    """[n][192] float64 features (before BF16 rounding) of [n][4] inputs:
    columns 32 d + 2 k, 32 d + 2 k + 1 = (sin, cos)(pi 2^(k/3) x_d), columns
    128..133 = the scaled inputs and lambda / 15, eta / 225, the rest zero."""
    x = np.asarray(inputs, np.float64)
    al, be, a, ct = x[:, 0], x[:, 1], x[:, 2], x[:, 3]
    xs = np.stack([al / 15.0, be / 15.0, 2.0 * a - 1.0, 2.0 * ct - 1.0], 1)
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    lam = -al * st
    eta = be * be + (al * al - a * a) * ct * ct
    F = np.zeros((x.shape[0], 192))
    for d in range(4):
        for k in range(16):
            arg = np.pi * FREQ[k].astype(np.float64) * xs[:, d]
            F[:, 32 * d + 2 * k] = np.sin(arg)
            F[:, 32 * d + 2 * k + 1] = np.cos(arg)
    F[:, 128:132] = xs
    F[:, 132] = lam / 15.0
    F[:, 133] = eta / 225.0
    return F


def unpack(params: np.ndarray):
    Ws, bs, off = [], [], 0
    for k, n in zip(LAYER_K, LAYER_N):
        Ws.append(np.asarray(params[off:off + n * k], np.float64).reshape(n, k))
        off += n * k
        bs.append(np.asarray(params[off:off + n], np.float64))
        off += n
    return Ws, bs


def silu(y):
    return y / (1.0 + np.exp(-y))


def silu_grad(y):
    s = 1.0 / (1.0 + np.exp(-y))
    return s * (1.0 + y * (1.0 - s))


def forward(params, F, emulate=True):
    """Head outputs and the cache the backward pass needs."""
    Ws, bs = unpack(params)
    if emulate == "f16":
        r = f16
    else:
        r = bf16 if emulate else (lambda v: np.asarray(v, np.float64))
    Wq = [r(W) for W in Ws]
    X = r(F)
    cache = {"X": [X], "Y": []}
    for l in range(4):
        Y = X @ Wq[l].T + bs[l]
        X = r(silu(Y))
        cache["Y"].append(Y)
        cache["X"].append(X)
    out = X @ Wq[4].T + bs[4]
    cache["Wq"] = Wq
    return out, cache


def reg_mask(j, cls, nc):
    if j <= 2 or j == 6:
        return nc >= 1
    if j <= 5:
        return nc >= 2
    return cls == 2


def loss_and_grad(out, targets):
    """Sum of losses (as the GPU's loss4) and dLoss/dout of the batch mean."""
    B = out.shape[0]
    t = np.asarray(targets, np.float64)
    cls = t[:, 0].astype(int)
    nc = t[:, 1].astype(int)
    d = np.zeros_like(out)
    used = cls >= 0
    lg = out[:, 0:3]
    m = lg.max(1, keepdims=True)
    e = np.exp(lg - m)
    Z = e.sum(1, keepdims=True)
    p = e / Z
    onehot = np.zeros_like(p)
    onehot[np.arange(B)[used], cls[used]] = 1.0
    ce = -(lg[np.arange(B), np.clip(cls, 0, 2)] - m[:, 0] - np.log(Z[:, 0]))
    d[:, 0:3] = np.where(used[:, None], (p - onehot) / B, 0.0)
    reg = 0.0
    for j in range(10):
        mk = reg_mask(j, cls, nc)
        err = out[:, 3 + j] - t[:, 2 + j]
        reg += float(np.sum(np.where(mk, err * err, 0.0)))
        d[:, 3 + j] = np.where(mk, 2.0 * err / B, 0.0)
    correct = float(np.sum(used & (np.argmax(lg, 1) == cls)))
    loss4 = np.array([float(np.sum(np.where(used, ce, 0.0))), reg, correct, float(used.sum())])
    return loss4, d


def backward(params, cache, dout, emulate=True):
    """Flat gradient (same layout as the parameters)."""
    r = bf16 if emulate else (lambda v: np.asarray(v, np.float64))
    Wq = cache["Wq"]
    X = cache["X"]
    Y = cache["Y"]
    gW, gb = [None] * 5, [None] * 5
    D = r(dout)
    gW[4] = D.T @ X[4]
    gb[4] = D.sum(0)
    dY = r((D @ Wq[4]) * silu_grad(Y[3]))
    for l in range(3, -1, -1):
        gW[l] = dY.T @ X[l]
        gb[l] = dY.sum(0)
        if l == 0:
            break
        dY = r((dY @ Wq[l]) * silu_grad(Y[l - 1]))
    flat = []
    for l in range(5):
        flat.append(gW[l].ravel())
        flat.append(gb[l])
    return np.concatenate(flat)


def total_loss(params, F, targets, emulate=False):
    out, _ = forward(params, F, emulate)
    loss4, _ = loss_and_grad(out, targets)
    B = F.shape[0]
    return (loss4[0] + loss4[1]) / B
