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
