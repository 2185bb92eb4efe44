"""The algorithmic FLOPs per accepted step that bench.py divides by are the
oracle's own counts (counting scalar: add, mul, div, sqrt count 1 each) over
seeded pixels of each workload."""
from __future__ import annotations

import math

import numpy as np
import pytest


def mean_flops_per_step(oracle, scenes, samples_per_scene, seed):
    rng = np.random.default_rng(seed)
    flops = steps = 0
    for s in scenes:
        for _ in range(samples_per_scene):
            al, be = rng.uniform(-12, 12, 2)
            _, st, c = oracle.count_ops(s, float(al), float(be))
            flops += c["add"] + c["mul"] + c["div"] + c["sqrt"]
            steps += st
    return flops / steps


def test_dp45_flops_constant(oracle):
    import bench

    scenes = bench.scenes_for("disk16", 0)
    f = mean_flops_per_step(oracle, scenes, 12, seed=1)
    assert f == pytest.approx(bench.FLOPS_PER_STEP["dp45"], rel=0.05)


def test_rk4_flops_constant(oracle):
    import bench

    scenes = bench.scenes_for("c0_256", 0)
    f = mean_flops_per_step(oracle, scenes, 60, seed=2)
    assert f == pytest.approx(bench.FLOPS_PER_STEP["rk4"], rel=0.05)


def test_rhs_operation_count(oracle):
    rhs, step = oracle.count_step_ops(spin=0.9, alpha=3.0, beta=2.0)
    # one right-hand side: 12 add, 13 mul, 2 div; one RK4 step: 4 of them + combination
    assert (rhs["add"], rhs["mul"], rhs["div"]) == (12, 13, 2)
    assert step["add"] + step["mul"] + step["div"] == 184
    assert math.isclose(step["div"], 10)


def test_transfer_flops_constant(oracle, lib):
    """FLOPs per accepted step of the volumetric transfer (c2_512: DP45 step
    plus its medium samples), counted over seeded pixels of the frame."""
    import ctypes as C_

    import bench
    from blackhole_b200 import rt
    from blackhole_b200._abi import default_scene
    from oracle import grmhd_oracle

    cells = grmhd_oracle.grid(128, 64, 64, 2.0, 50.0)
    desc = rt.SynchrotronLut(None, 256, 256, math.log(0.1), math.log(1000.0), math.log(1e-4), math.log(1e4))
    tab = np.empty((256, 256), np.float32)
    rt._lib()
    assert lib.bh_synchrotron_lut_host(C_.byref(desc), tab.ctypes.data) == 0
    s = default_scene(width=512, height=512, spin=0.94, theta_obs=math.radians(17.0), integrator=1,
                      max_crossings=1, precision=0)
    s.max_steps = 2000
    s.alpha_min, s.alpha_max, s.beta_min, s.beta_max = -20.0, 20.0, -20.0, 20.0
    p = rt.rt_defaults()
    pix = np.random.default_rng(3).integers(0, 512 * 512, 400)
    c = oracle.count_rt_ops(s, cells, (2.0, 50.0), tab, (desc.log_theta_min, desc.log_theta_max),
                            (desc.log_x_min, desc.log_x_max), p.nu_hz, p.length_cm, p.ds_max, p.min_transmit, pix)
    f = (c["add"] + c["mul"] + c["div"] + c["sqrt"]) / c["steps"]
    assert f == pytest.approx(bench.FLOPS_PER_STEP["rt"], rel=0.05)


def test_surrogate_flop_constants(lib):
    """The network FLOPs the surrogate line divides by follow the library's
    layer shapes: 134 used input features of 192 (the rest is zero padding),
    4 hidden layers of 256, a 16-wide head. The kernel executes the input
    layer on 144 columns (two 64-column K chunks and the first 16-column K
    step of the third, which holds features 128..133)."""
    import bench

    K = [192, 256, 256, 256, 256]
    N = [256, 256, 256, 256, 16]
    assert lib.bh_surrogate_param_count() == sum(k * n + n for k, n in zip(K, N))
    used = [134] + K[1:]
    assert bench.SURROGATE_FLOPS_PER_RAY == 2.0 * sum(k * n for k, n in zip(used, N))
    executed_k0 = 128 + 16 * math.ceil((134 - 128) / 16)
    assert executed_k0 == 144
    assert bench.SURROGATE_MMA_FLOPS_PER_RAY == 2.0 * sum(k * n for k, n in zip([executed_k0] + K[1:], N))
