"""The Stokes-step oracle against the reference's known answers and against
an independent solution (matrix exponential), on the CPU.

Known answers: the reference's tests/cuda_stokes_test.cu:180-330 (pure
rotation, pure absorption, the polarization bound along a sequence of
emitting steps, a rotation and its inverse, zero input)."""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))
import stokes_oracle as SO  # noqa: E402


def test_pure_rotation():
    r = SO.stokes_step([1.0, 1.0, 0.0, 0.0], 0, 0, 0, 0, 0.0, math.pi / 4, 1.0)
    np.testing.assert_allclose(r, [1.0, math.cos(math.pi / 4), math.sin(math.pi / 4), 0.0], atol=1e-12)


def test_pure_absorption():
    r = SO.stokes_step([1.0, 0.6, 0.3, 0.1], 0, 0, 0, 0, 2.0, 0.0, 0.5)
    np.testing.assert_allclose(r, np.array([1.0, 0.6, 0.3, 0.1]) * math.exp(-1.0), rtol=1e-12)


def test_rotation_round_trip():
    s = SO.stokes_step([1.0, 1.0, 0.0, 0.0], 0, 0, 0, 0, 0.0, 0.7, 1.0)
    r = SO.stokes_step(s, 0, 0, 0, 0, 0.0, -0.7, 1.0)
    np.testing.assert_allclose(r, [1.0, 1.0, 0.0, 0.0], atol=1e-12)


def test_zero_input_stays_zero():
    for a, rho in ((0.0, 0.0), (1.5, 0.0), (0.0, 2.0), (0.3, 0.8)):
        np.testing.assert_array_equal(SO.stokes_step([0, 0, 0, 0], 0, 0, 0, 0, a, rho, 0.7), [0, 0, 0, 0])


def test_polarization_bound_along_emitting_steps():
    """|P| <= I after every step when the emission is itself physical
    (jQ^2 + jU^2 + jV^2 <= jI^2), from an unpolarized start."""
    rng = np.random.default_rng(5)
    s = np.zeros(4)
    for _ in range(2000):
        jI = rng.uniform(0.0, 2.0)
        d = rng.normal(size=3)
        jpol = jI * rng.uniform(0.0, 1.0) * d / np.linalg.norm(d)
        s = SO.stokes_step(s, jI, *jpol, rng.uniform(0.0, 2.0), rng.uniform(-3.0, 3.0), rng.uniform(0.0, 0.5))
        assert s[0] >= 0.0
        assert s[1] ** 2 + s[2] ** 2 + s[3] ** 2 <= s[0] ** 2 * (1 + 1e-12) + 1e-24


@pytest.mark.parametrize("seed", range(4))
def test_restatement_matches_matrix_exponential(seed):
    rng = np.random.default_rng(seed)
    for _ in range(300):
        s = rng.normal(size=4)
        j = rng.normal(size=4)
        a = float(rng.choice([0.0, rng.uniform(0.0, 5.0)]))
        rho = float(rng.choice([0.0, rng.uniform(-4.0, 4.0)]))
        ds = float(rng.uniform(1e-6, 2.0))
        want = SO.stokes_step_expm(s, *j, a, rho, ds)
        got = SO.stokes_step(s, *j, a, rho, ds)
        # the reference's scalar channels are first order in tau below 1e-4
        tol = 1e-9 if a * ds < 1e-4 else 1e-11
        np.testing.assert_allclose(got, want, rtol=tol, atol=tol * (1 + np.abs(s).sum() + np.abs(j).sum() * ds))


def test_reference_formula_cancels_for_tiny_absorption_and_rotation():
    """A quirk of the reference's step, kept by the restatement: with alpha_I
    and rho_V both tiny but nonzero (A^2 + R^2 above its 1e-60 pure-emission
    threshold, neither 1e15 times the other), its closed form divides a
    cancelled difference by A^2 + R^2, and the (Q, U) source terms are lost.
    The library's step switches to the Taylor series there
    (test_gpu_legacy_volume.py checks it against the exact solution)."""
    s, j = [0.0, 0.0, 0.0, 0.0], [1.0, 0.5, -0.4, 0.2]
    exact = SO.stokes_step_expm(s, *j, 1e-20, 1e-20, 1.0)
    ref = SO.stokes_step(s, *j, 1e-20, 1e-20, 1.0)
    np.testing.assert_allclose(exact, [1.0, 0.5, -0.4, 0.2], rtol=1e-12)
    assert abs(ref[1] - exact[1]) > 0.1 or abs(ref[2] - exact[2]) > 0.1
