"""Batches: frames of uneven size, spin, inclination and observer radius
traced by one persistent launch (BH_KerrBatch), with CUDA-graph replay,
per-frame completion times and the launch-shape autotuner.

A batch performs the same per-pixel arithmetic as single-frame traces: in
FP64 the outputs are bit-identical to the oracle; in mixed precision they
agree with the single-frame mixed kernel to FP32 rounding.
"""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from test_gpu_image import ULP_FIELDS, assert_bitexact, gpu_trace, scene

pytestmark = pytest.mark.gpu


def uneven_scenes(precision=0, integrator=1, seed=5):
    rng = np.random.default_rng(seed)
    sizes = [(17, 9), (64, 48), (1, 1), (33, 33), (0, 7), (40, 25), (3, 61)]
    out = []
    for w, h in sizes:
        out.append(scene(width=w, height=h, spin=float(rng.uniform(0, 0.998)),
                         theta_obs=math.radians(float(rng.uniform(5, 89))),
                         r_obs=float(math.exp(rng.uniform(math.log(100), math.log(5000)))),
                         integrator=integrator, precision=precision, max_crossings=int(rng.integers(1, 4))))
    return out


def host(outs):
    return [{k: v.cpu().numpy() for k, v in o.items()} for o in outs]


def test_fp64_batch_bitexact_vs_oracle(cuda, oracle):
    from blackhole_b200 import kerr

    scenes = uneven_scenes()
    b = kerr.TraceBatch(scenes)
    b.trace()
    torch.cuda.synchronize()
    for s, got in zip(scenes, host(b.outs)):
        if s.width * s.height == 0:
            continue
        assert_bitexact(got, oracle.trace_pixels(s))


def test_rk4_batch_bitexact_vs_single_frame(cuda):
    from blackhole_b200 import kerr

    scenes = uneven_scenes(integrator=0, seed=9)[:4]
    b = kerr.TraceBatch(scenes)
    b.trace()
    torch.cuda.synchronize()
    for s, got in zip(scenes, host(b.outs)):
        single = gpu_trace(s)
        for k in got:
            np.testing.assert_array_equal(got[k], single[k], err_msg=k)


def test_mixed_batch_matches_single_frame_mixed(cuda):
    from blackhole_b200 import kerr

    scenes = uneven_scenes(precision=1)
    b = kerr.TraceBatch(scenes)
    b.trace()
    torch.cuda.synchronize()
    for s, got in zip(scenes, host(b.outs)):
        if s.width * s.height == 0:
            continue
        single = gpu_trace(s)
        assert np.mean(got["cls"] == single["cls"]) >= 0.999
        same = (got["n_cross"] == single["n_cross"]) & (got["n_cross"] > 0)
        np.testing.assert_allclose(got["g"][0][same], single["g"][0][same], rtol=1e-6)


def test_graph_replay_and_frame_times(cuda):
    from blackhole_b200 import kerr

    scenes = uneven_scenes(precision=1)
    b = kerr.TraceBatch(scenes)
    st = torch.cuda.Stream()
    b.trace(stream=st)
    st.synchronize()
    ref = host(b.outs)
    for _ in range(3):
        for o in b.outs:
            for v in o.values():
                v.zero_()
        b.trace_graph(stream=st)
        st.synchronize()
        for a, r in zip(host(b.outs), ref):
            for k in a:
                np.testing.assert_array_equal(a[k], r[k], err_msg=k)
    t = b.frame_times()
    sizes = np.array([s.width * s.height for s in scenes])
    assert (t[sizes > 0] > 0).all() and (t[sizes == 0] == 0).all()
    assert np.isfinite(t).all() and t.max() < 60_000


def test_autotune_keeps_results(cuda):
    from blackhole_b200 import kerr

    scenes = [scene(width=96, height=96, spin=a, integrator=1, precision=1) for a in (0.1, 0.6, 0.95)]
    b = kerr.TraceBatch(scenes)
    b.trace()
    torch.cuda.synchronize()
    ref = host(b.outs)
    cfg = b.autotune(max_pixels=20_000)
    assert cfg["block_threads"] in (64, 128) and cfg["ctas_per_sm"] >= 1 and cfg["refill_steps"] in (1, 2, 4)
    assert b.launch() == cfg
    b.trace()
    torch.cuda.synchronize()
    for a, r in zip(host(b.outs), ref):
        for k in a:
            np.testing.assert_array_equal(a[k], r[k], err_msg=k)


@pytest.mark.parametrize("block,per_sm,refill", [(32, 1, 1), (64, 2, 3), (128, 0, 8)])
def test_launch_shapes_do_not_change_results(cuda, block, per_sm, refill):
    from blackhole_b200 import kerr

    scenes = uneven_scenes(seed=11)
    b = kerr.TraceBatch(scenes)
    b.trace()
    torch.cuda.synchronize()
    ref = host(b.outs)
    b.set_launch(block, per_sm, refill)
    b.trace()
    torch.cuda.synchronize()
    for a, r in zip(host(b.outs), ref):
        for k in a:
            np.testing.assert_array_equal(a[k], r[k], err_msg=k)


def test_batch_rejects_mixed_integrators(cuda):
    from blackhole_b200 import kerr

    with pytest.raises(RuntimeError, match="share integrator"):
        kerr.TraceBatch([scene(width=4, height=4, integrator=0), scene(width=4, height=4, integrator=1)])
