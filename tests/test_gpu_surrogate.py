"""GPU checks of the surrogate network's tensor-core kernels.

* the BF16 GEMM (tcgen05, FP32 accumulation) against a float64 product of
  the same BF16 operands, for every tile width and split-K path it serves;
* features, forward pass and the full gradient (forward, loss, backward,
  split-K weight gradients, bias sums) against the CPU oracle, which rounds
  to BF16 at the points where the GPU stores BF16;
* training targets built from the integrator's own outputs;
* a short training run on traced rays lowers the loss.
"""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from oracle import surrogate_oracle as so

pytestmark = pytest.mark.gpu


def rand_inputs(n, seed):
    g = torch.Generator().manual_seed(seed)
    u = torch.rand(n, 4, generator=g, dtype=torch.float64)
    x = torch.empty(n, 4, dtype=torch.float64)
    x[:, 0] = -15 + 30 * u[:, 0]
    x[:, 1] = -15 + 30 * u[:, 1]
    x[:, 2] = 0.998 * u[:, 2]
    x[:, 3] = torch.cos(torch.deg2rad(5 + 84 * u[:, 3]))
    return x.float()


@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (300, 256, 192), (1000, 16, 256), (257, 192, 1024),
                                   (128, 512, 128), (4096, 256, 256)])
def test_bf16_gemm_matches_float64(cuda, M, N, K):
    from blackhole_b200 import surrogate as S

    g = torch.Generator().manual_seed(M * 7 + N + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, generator=g).to(torch.bfloat16)
    ref = A.double() @ B.double().T
    got = S.bf16_gemm(A.cuda(), B.cuda()).double().cpu()
    torch.cuda.synchronize()
    err = (got - ref).abs().max().item()
    assert err <= 1e-5 * math.sqrt(K) * ref.abs().max().item(), err


def test_features_match_oracle(cuda):
    from blackhole_b200 import surrogate as S

    x = rand_inputs(777, 1)
    F = S.features(x.cuda()).float().cpu().numpy().astype(np.float64)
    ref = so.bf16(so.features(x.double().numpy()))
    tol = 2.0 ** -7 * np.abs(ref) + 1e-5  # 1 BF16 ulp; angle doubling keeps sin/cos within ~2e-6
    assert np.all(np.abs(F - ref) <= tol)
    assert np.mean(F == ref) > 0.999


def test_forward_matches_oracle(cuda):
    """The fused inference kernel evaluates the network in FP16 (weights,
    features, activations; FP32 accumulation): against the oracle rounding
    to FP16 at the same points it agrees to the MUFU tanh's ~2^-11, and it
    stays within BF16 noise of the training path's BF16 evaluation."""
    from blackhole_b200 import surrogate as S

    net = S.Surrogate(max_batch=1024, seed=5)
    x = rand_inputs(1000, 2).cuda()
    head = net.forward(x).double().cpu().numpy()
    F = so.features(x.double().cpu().numpy())
    params = net.get_params().astype(np.float64)
    ref, _ = so.forward(params, F, emulate="f16")
    assert net.device_error() == 0
    rel = np.linalg.norm(head - ref) / np.linalg.norm(ref)
    assert rel < 2e-3, rel
    ref_bf16, _ = so.forward(params, so.bf16(F), emulate=True)
    rel = np.linalg.norm(head - ref_bf16) / np.linalg.norm(ref_bf16)
    assert rel < 1e-2, rel


def synthetic_targets(B, seed):
    rng = np.random.default_rng(seed)
    t = np.zeros((B, 16), np.float32)
    cls = rng.integers(0, 3, B)
    nc = np.where(cls == 1, rng.integers(1, 3, B), 0)
    t[:, 0], t[:, 1] = cls, nc
    t[:, 2:12] = rng.normal(0.0, 0.5, (B, 10))
    return t


def test_gradients_match_oracle(cuda):
    from blackhole_b200 import surrogate as S

    B = 512
    net = S.Surrogate(max_batch=B, seed=7)
    x = rand_inputs(B, 3).cuda()
    t = synthetic_targets(B, 4)
    grad, loss = net.gradients(x, torch.from_numpy(t).cuda())
    grad = grad.double().cpu().numpy()
    loss = loss.cpu().numpy()
    assert net.device_error() == 0
    params = net.get_params().astype(np.float64)
    F = S.features(x).float().cpu().numpy().astype(np.float64)
    out, cache = so.forward(params, F, emulate=True)
    loss_ref, dout = so.loss_and_grad(out, t.astype(np.float64))
    ref = so.backward(params, cache, dout, emulate=True)
    np.testing.assert_allclose(loss, loss_ref, rtol=2e-3)
    for l, (ws, bs) in enumerate(S.weight_slices()):
        for name, sl in (("W", ws), ("b", bs)):
            rel = np.linalg.norm(grad[sl] - ref[sl]) / max(np.linalg.norm(ref[sl]), 1e-30)
            assert rel < 1e-2, (l, name, rel)


def test_make_targets_from_traced_rays(cuda):
    from blackhole_b200 import kerr
    from blackhole_b200 import surrogate as S

    s = kerr.scene(width=48, height=40, spin=0.9, theta_obs=math.radians(75), integrator=1, precision=0,
                   max_crossings=2, alpha_min=-15, alpha_max=15, beta_min=-15, beta_max=15)
    o = kerr.trace_image(s)
    n = s.width * s.height
    tg = S.make_targets(o, n, 2).cpu().numpy()
    h = {k: v.cpu().numpy() for k, v in o.items()}
    nc = np.minimum(h["n_cross"], 2)
    oc = np.where(nc >= 1, 1, np.where(h["cls"] == 0, 0, np.where(h["cls"] == 2, 2, -1)))
    np.testing.assert_array_equal(tg[:, 0], oc)
    np.testing.assert_array_equal(tg[:, 1], nc)
    d1 = nc >= 1
    np.testing.assert_allclose(tg[d1, 2], np.log(h["r_hit"][0][d1]) - 2, rtol=1e-6)
    np.testing.assert_allclose(tg[d1, 8], h["g"][0][d1] - 1, rtol=1e-5, atol=1e-7)
    d2 = nc >= 2
    assert d2.any()
    np.testing.assert_allclose(tg[d2, 5], np.log(h["r_hit"][1][d2]) - 2, rtol=1e-6)
    esc = oc == 2
    np.testing.assert_allclose(tg[esc, 9], np.cos(h["theta_inf"][esc]), rtol=1e-5, atol=1e-6)
    inp = S.grid_inputs(s).cpu().numpy()
    al = -15 + (np.arange(n) % 48 + 0.5) * 30 / 48
    np.testing.assert_allclose(inp[:, 0], al, rtol=1e-6)


def test_short_training_run_lowers_loss(cuda):
    from blackhole_b200 import surrogate as S

    data = S.generate_rays(n_frames=16, size=64, seed=11)
    assert data.inputs.shape == (16 * 64 * 64, 4)
    net = S.Surrogate(max_batch=4096, seed=1)
    hist = S.train(net, data, epochs=12, batch=4096, lr=2e-3, log_every=16, log=None)
    assert net.device_error() == 0
    first, last = hist[0], hist[-1]
    assert last["ce"] < 0.5 * first["ce"], hist
    assert last["acc"] > 0.9, hist
