"""GPU parity of the batched reference src/physics API against the reference.

bh_kerr_potentials / bh_kerr_step_mino / bh_kerr_trace_rays restate
physics::kerrPotentials, kerrStepMino and KerrRaytracer::trace
(src/physics/kerr.cpp:40-134, src/physics/raytracer.h:324-378) in FP64 with
no FMA contraction; the golden vectors come from the reference's own compiled
kerr.cpp. The only arithmetic difference is CUDA's sin/cos against glibc's
(an ulp or two), hence the small relative tolerances, which grow with the
number of steps taken.
"""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from conftest import load_golden
from test_oracle_pins import TRACE_TAGS, trace_case

pytestmark = pytest.mark.gpu

FIELDS = ("r", "theta", "phi", "t", "sign_r", "sign_theta")


def dev(x):
    return torch.as_tensor(np.ascontiguousarray(x, np.float64), device="cuda")


@pytest.mark.parametrize("tag", ["geom", "cgs"])
def test_potentials_and_step_vs_reference(cuda, tag):
    from blackhole_b200 import kerr

    g = load_golden("kerr_step_ref.npz")
    mass, a = float(g[f"{tag}_mass"]), float(g[f"{tag}_a"])
    e, lz, q = dev(g[f"{tag}_e"]), dev(g[f"{tag}_lz"]), dev(g[f"{tag}_q"])
    st = {k: dev(g[f"{tag}_in_{k}"]) for k in FIELDS}
    pot = kerr.kerr_potentials(st["r"], st["theta"], mass, a, e, lz, q)
    for k in ("r_pot", "dr_pot", "theta_pot", "dtheta_pot"):
        ref = g[f"{tag}_pot_{k}"]
        scale = np.abs(ref) + 1e-300
        got = pot[k].cpu().numpy()
        # relative to the size of the largest term of each potential
        assert np.all(np.abs(got - ref) <= 1e-12 * np.maximum(scale, np.abs(ref).max() * 1e-6)), k
    dlam = dev(g[f"{tag}_dlam"])
    one = {k: v.clone() for k, v in st.items()}
    kerr.kerr_step_mino(one, mass, a, e, lz, q, dlam)
    hundred = {k: v.clone() for k, v in st.items()}
    for _ in range(100):
        kerr.kerr_step_mino(hundred, mass, a, e, lz, q, dlam)
    torch.cuda.synchronize()
    for k in ("r", "theta", "phi", "t"):
        np.testing.assert_allclose(one[k].cpu().numpy(), g[f"{tag}_step1_{k}"], rtol=1e-13, atol=1e-300, err_msg=k)
        np.testing.assert_allclose(hundred[k].cpu().numpy(), g[f"{tag}_step100_{k}"], rtol=1e-10, atol=1e-300,
                                   err_msg=k)


def test_step_scalar_dlam_matches_array(cuda):
    from blackhole_b200 import kerr

    g = load_golden("kerr_step_ref.npz")
    mass, a = float(g["geom_mass"]), float(g["geom_a"])
    e, lz, q = dev(g["geom_e"]), dev(g["geom_lz"]), dev(g["geom_q"])
    s1 = {k: dev(g[f"geom_in_{k}"]) for k in FIELDS}
    s2 = {k: v.clone() for k, v in s1.items()}
    kerr.kerr_step_mino(s1, mass, a, e, lz, q, 1e-3)
    kerr.kerr_step_mino(s2, mass, a, e, lz, q, dev(np.full(len(g["geom_e"]), 1e-3)))
    for k in FIELDS:
        assert torch.equal(s1[k], s2[k])


@pytest.mark.parametrize("tag", TRACE_TAGS)
def test_trace_rays_vs_reference(cuda, tag):
    from blackhole_b200 import kerr

    g = load_golden("kerr_trace_ref.npz")
    (mass, a, r_h, r_esc, step, max_steps), eq, gen = trace_case(g, tag)
    tr = kerr.KerrRaytracer(mass, a)
    tr.set_step_size(step)
    tr.set_escape_radius(r_esc)
    tr.set_max_steps(max_steps)
    assert tr.params.r_horizon == r_h
    for kind, (st, e, lz, q) in (("eq", eq), ("gen", gen)):
        res = tr.trace({k: dev(v) for k, v in st.items()}, dev(e), dev(lz), dev(q))
        torch.cuda.synchronize()
        status = res.status.cpu().numpy()
        steps = res.steps_taken.cpu().numpy()
        ref_status, ref_steps = g[f"{tag}_{kind}_status"], g[f"{tag}_{kind}_steps"]
        # sin/cos ulps can move a ray across a termination test only by one
        # step at most; the outcome class must agree
        np.testing.assert_array_equal(status, ref_status, err_msg=f"{kind} status")
        assert np.all(np.abs(steps - ref_steps) <= 1), kind
        same = steps == ref_steps
        final = [("r", res.final_r), ("theta", res.final_theta)]
        if tag.startswith("geom"):
            # The CGS cases use the reference constructor's Mino step (0.02 r_s),
            # with which every ray jumps out in one step and its stage states
            # reach theta ~ 1e8 rad; there sin^2 theta is near the 1e-12 clamp
            # and phi inherits the sin/cos ulp differences at full scale.
            final.append(("phi", res.final_phi))
        for k, ours in final:
            np.testing.assert_allclose(ours.cpu().numpy()[same], g[f"{tag}_{kind}_{k}"][same], rtol=1e-7,
                                       err_msg=f"{kind} {k}")


def test_raytracer_defaults_match_reference_constructor(lib):
    from blackhole_b200 import kerr

    g = load_golden("kerr_trace_ref.npz")
    for spin_tag in ("a0", "a09"):
        tag = f"cgs_{spin_tag}"
        mass = float(g[f"{tag}_mass"])
        tr = kerr.KerrRaytracer(mass, float(g[f"{tag}_a"]))
        assert tr.params.r_horizon == float(g[f"{tag}_r_horizon"])
        assert tr.params.r_escape == float(g[f"{tag}_r_escape"])
        assert tr.params.step_size == float(g[f"{tag}_step_size"])
        assert tr.params.max_steps == 10000


def test_reference_turning_point_stall_reproduced(cuda):
    """The drop-in keeps the reference's first-order scheme, including its
    stall at radial turning points (equatorial b = 16M ray from r = 100)."""
    from blackhole_b200 import kerr

    mass = 2.99792458e10**2 / 6.67430e-8
    tr = kerr.KerrRaytracer(mass, 0.0)
    tr.set_step_size(2e-4)
    tr.set_max_steps(20000)
    st = {k: dev([v]) for k, v in dict(r=100.0, theta=0.5 * math.pi, phi=0.0, t=0.0, sign_r=-1.0,
                                        sign_theta=1.0).items()}
    res = tr.trace(st, dev([1.0]), dev([16.0]), dev([0.0]))
    assert int(res.status[0]) == 4
    assert 14.0 < float(res.final_r[0]) < 16.0
