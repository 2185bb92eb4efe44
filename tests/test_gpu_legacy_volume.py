"""The render calls' volumetric modes (BH_LaunchParams.rte_enabled,
stokes_enabled): the Stokes transfer step against its analytic limits and the
exact solution, and the composited frames against the properties the model
guarantees.

The step's known answers are the reference's (tests/cuda_stokes_test.cu:
180-330): pure rotation, pure absorption, the polarization bound, a rotation
round trip, zero input, no NaN. The exact solution is the oracle's matrix
exponential (oracle/stokes_oracle.py), pinned on the CPU
(tests/test_stokes_oracle.py).

The frames cannot be compared with the reference's own kernel: for a
spinning hole its Kerr path traces the time-reversed photon (a mirror
image), and for a = 0 both fall back to the single-scatter look. So the
checks are the model's:
* a = 0: the RTE and Stokes modes give the single-scatter frame exactly;
* with disk emission off and no ring glow, the RTE frame is the
  single-scatter sky (the slab is empty, so the transmittance stays 1);
* emission only falls as the opacity rises (each segment's j (1 - e^-tau) /
  alpha is at most j ds, and the transmittance in front of it at most 1);
* Stokes with field angle 0 and no Faraday rotation emits Q < 0, U = 0 and
  no V, so the tint lowers red only: green and blue equal the RTE frame's.
"""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import stokes_oracle as SO  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def leg():
    from blackhole_b200 import legacy

    legacy.library()
    before = legacy.get_shading()
    legacy.set_shading(legacy.SHADING_REFERENCE)
    yield legacy
    legacy.set_shading(before)


def steps(leg, state, coef):
    s = torch.tensor(np.asarray(state, dtype=np.float32).reshape(-1, 4), device="cuda")
    c = torch.tensor(np.asarray(coef, dtype=np.float32).reshape(-1, 7), device="cuda")
    out = leg.stokes_steps(s, c)
    torch.cuda.synchronize()
    return out.cpu().numpy().astype(np.float64)


def test_known_answers(cuda, leg):
    r = steps(leg, [[1, 1, 0, 0], [1, 0.6, 0.3, 0.1], [0, 0, 0, 0]],
              [[0, 0, 0, 0, 0, math.pi / 4, 1.0], [0, 0, 0, 0, 2.0, 0, 0.5], [0, 0, 0, 0, 0.3, 0.8, 0.7]])
    np.testing.assert_allclose(r[0], [1, math.cos(math.pi / 4), math.sin(math.pi / 4), 0], atol=1e-6)
    np.testing.assert_allclose(r[1], np.array([1, 0.6, 0.3, 0.1]) * math.exp(-1), rtol=1e-6)
    np.testing.assert_array_equal(r[2], [0, 0, 0, 0])
    back = steps(leg, r[0], [0, 0, 0, 0, 0, -math.pi / 4, 1.0])
    np.testing.assert_allclose(back[0], [1, 1, 0, 0], atol=1e-6)


def test_matches_exact_solution(cuda, leg):
    rng = np.random.default_rng(11)
    n = 4096
    s = rng.normal(size=(n, 4))
    j = rng.normal(size=(n, 4))
    a = np.where(rng.random(n) < 0.2, 0.0, rng.uniform(0, 5, n))
    rho = np.where(rng.random(n) < 0.2, 0.0, rng.uniform(-4, 4, n))
    tiny = rng.random(n) < 0.1  # both tiny: the reference's closed form cancels here
    a[tiny], rho[tiny] = 1e-20, 1e-20
    ds = rng.uniform(1e-6, 2.0, n)
    coef = np.column_stack([j, a, rho, ds])
    got = steps(leg, s, coef)
    want = np.array([SO.stokes_step_expm(s[k], *j[k], a[k], rho[k], ds[k]) for k in range(n)])
    scale = 1 + np.abs(s).sum(1) + np.abs(j).sum(1) * ds
    err = np.abs(got - want).max(1) / scale
    assert err.max() < 2e-6, err.max()


def test_ds_zero_and_negative_absorption(cuda, leg):
    r = steps(leg, [[0.3, 0.1, -0.2, 0.05]] * 2, [[1, 1, 1, 1, 1, 1, 0.0], [1, 0, 0, 0, -5.0, 0, 1.0]])
    np.testing.assert_array_equal(r[0], np.float32([0.3, 0.1, -0.2, 0.05]))
    np.testing.assert_allclose(r[1], [1.3, 0.1, -0.2, 0.05], rtol=1e-6)  # alpha < 0 counts as 0


def test_polarization_bound_and_no_nan(cuda, leg):
    rng = np.random.default_rng(3)
    chains = 512
    state = torch.zeros(chains, 4, device="cuda")
    for _ in range(300):
        jI = rng.uniform(0, 2, chains)
        d = rng.normal(size=(chains, 3))
        jpol = (jI * rng.uniform(0, 1, chains))[:, None] * d / np.linalg.norm(d, axis=1, keepdims=True)
        coef = np.column_stack([jI, jpol, rng.uniform(0, 2, chains), rng.uniform(-3, 3, chains),
                                rng.uniform(0, 0.5, chains)]).astype(np.float32)
        state = leg.stokes_steps(state, torch.tensor(coef, device="cuda"))
    s = state.cpu().numpy().astype(np.float64)
    assert np.all(np.isfinite(s)) and np.all(s[:, 0] >= 0)
    assert np.all(s[:, 1] ** 2 + s[:, 2] ** 2 + s[:, 3] ** 2 <= s[:, 0] ** 2 * (1 + 1e-4) + 1e-10)


def test_bad_arguments(cuda, leg):
    with pytest.raises(ValueError):
        leg.stokes_steps(torch.zeros(3, 4, device="cuda"), torch.zeros(3, 6, device="cuda"))


def frame(leg, spin, rte=0, stokes=0, opacity=1.0, disk=1, glow=0.0, background=1, b_angle=0.0, ne=0.0):
    """A 128 x 96 bridge camera at 15 rs, 1.3 rad from the spin axis, aimed
    at the hole; steps of 0.04, 20,000 at most; LUTs off."""
    p = leg.bridge_params(spin, 15.0, 1.3, 0.6, 128, 96)
    p.step_size, p.max_steps = 0.04, 20000
    p.adisk_enabled, p.redshift_enabled, p.kerr_enabled, p.use_luts = disk, 1, 1, 0
    p.doppler_strength = 1.0
    p.photon_glow_strength = glow
    p.background_enabled = background
    p.background_intensity = 1.0 if background else 0.0
    p.adisk_lit = 1.0
    p.rte_enabled, p.rte_opacity_scale = rte, opacity
    p.stokes_enabled, p.stokes_b_field_angle, p.stokes_ne_scale = stokes, b_angle, ne
    fb = torch.zeros(p.width * p.height * 4, dtype=torch.float32, device="cuda")
    leg.launch(p, fb, 0)
    torch.cuda.synchronize()
    return fb.view(p.height, p.width, 4).cpu().numpy()


def test_no_spin_falls_back_to_single_scatter(cuda, leg):
    base = frame(leg, 0.0, glow=1.0)
    np.testing.assert_array_equal(frame(leg, 0.0, rte=1, glow=1.0), base)
    np.testing.assert_array_equal(frame(leg, 0.0, stokes=1, glow=1.0), base)


def test_empty_slab_leaves_the_sky(cuda, leg):
    sky = frame(leg, 0.9, disk=0)
    vol = frame(leg, 0.9, rte=1, disk=0)
    assert np.all(np.isfinite(vol)) and np.all(vol[..., 3] == 1.0)
    np.testing.assert_allclose(vol, sky, rtol=1e-5, atol=1e-7)


def test_emission_falls_as_opacity_rises(cuda, leg):
    tot = []
    for op in (0.0, 1.0, 30.0):
        img = frame(leg, 0.9, rte=1, opacity=op, background=0)
        assert np.all(np.isfinite(img)) and np.all(img[..., :3] >= 0.0)
        tot.append(float(img[..., :3].sum()))
    assert tot[0] > 0.0
    assert tot[0] >= tot[1] >= tot[2], tot
    assert tot[2] < tot[0]


def test_stokes_tint_lowers_red_only_without_rotation(cuda, leg):
    rte = frame(leg, 0.9, rte=1, background=0)
    sto = frame(leg, 0.9, stokes=1, background=0, b_angle=0.0, ne=0.0)
    lit = rte[..., :3].max(-1) > 0
    assert lit.mean() > 0.05
    np.testing.assert_allclose(sto[..., 1], rte[..., 1], rtol=1e-5, atol=1e-8)
    np.testing.assert_allclose(sto[..., 2], rte[..., 2], rtol=1e-5, atol=1e-8)
    assert np.all(sto[..., 0] <= rte[..., 0] * (1 + 1e-5) + 1e-8)
    assert np.mean(sto[..., 0][lit] < rte[..., 0][lit]) > 0.5
    # a field angle of 45 degrees moves the tint into green: U < 0, Q = 0
    sto45 = frame(leg, 0.9, stokes=1, background=0, b_angle=math.pi / 4, ne=0.0)
    assert np.mean(sto45[..., 1][lit] < rte[..., 1][lit]) > 0.5
