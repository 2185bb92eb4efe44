"""CPU pins of the radiative-transfer physics against the reference's own
compiled functions (src/physics/rte_integrator.h through oracle/_ref)."""
from __future__ import annotations

import math

import numpy as np

E, ME, C = 4.80320425e-10, 9.1093837015e-28, 2.99792458e10


def test_synchrotron_table_matches_reference_emissivity(lib, reflib):
    from blackhole_b200 import rt

    desc = rt.SynchrotronLut(None, 64, 96, math.log(0.1), math.log(1000.0), math.log(1e-4), math.log(1e4))
    tab = np.empty((64, 96), np.float32)
    rt._lib()
    import ctypes as C_

    assert lib.bh_synchrotron_lut_host(C_.byref(desc), tab.ctypes.data) == 0
    nu, n = 230e9, 1e5
    for i in range(0, 64, 7):
        th = math.exp(desc.log_theta_min + (desc.log_theta_max - desc.log_theta_min) * i / 63)
        for k in range(0, 96, 5):
            x = math.exp(desc.log_x_min + (desc.log_x_max - desc.log_x_min) * k / 95)
            nu_b = nu / (1.5 * x * th * th)
            b = nu_b * 2 * math.pi * ME * C / E
            ref = reflib.synchrotron_j(nu, b, n, th)
            got = math.exp(float(tab[i, k])) * n * nu_b  # the table holds ln(j / (n nu_B)) in FP32
            assert abs(got - ref) <= 1e-5 * abs(ref), (i, k, got, ref)


def test_absorption_is_kirchhoff_at_the_emitted_frequency(reflib):
    kb = 1.380649e-16
    for th in (0.5, 5.0, 50.0):
        for nu in (86e9, 230e9, 345e9):
            b, n = 20.0, 1e5
            j = reflib.synchrotron_j(nu, b, n, th)
            a = reflib.synchrotron_alpha(nu, b, n, th)
            bnu = reflib.planck(nu, th * ME * C * C / kb)
            assert abs(a - j / bnu) <= 1e-14 * abs(a)


def test_front_to_back_equals_reference_rte_path(oracle, reflib):
    rng = np.random.default_rng(4)
    for scale in (1e-16, 1e-9, 1e-6, 1e-3):  # optically thin to thick, both Taylor and exact branches
        j = rng.uniform(0, 1e-9, 200)
        a = scale * 10 ** rng.uniform(-2, 2, 200)
        a[::17] = 0.0  # pure emission segments
        ds = rng.uniform(1e5, 1e7, 200)
        got, ref = oracle.rt_path(j, a, ds), reflib.rte_path(j, a, ds)
        # The reference's tau < 1e-4 branch attenuates the incoming I to first
        # order in tau and adds S (1 - e^-tau) to second order; front to back
        # both are second order: they differ by O(tau^2) per thin segment.
        assert abs(got - ref) <= 1e-8 * abs(ref), (scale, got, ref)
