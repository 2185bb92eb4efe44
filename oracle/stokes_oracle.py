"""Oracle for the polarized transfer step of the render calls' Stokes mode.

Test infrastructure only: the parity tests, not the library, use it.

`stokes_step` restates the reference's d_stokes_step
(src/cuda/device_physics.cuh:2216-2284) in FP64 numpy, branch for branch:
scalar channels I and V with absorption alpha_I, (Q, U) with absorption and
Faraday rotation rho_V, each solved exactly over the segment ds.

`stokes_step_expm` solves the same linear system independently: the state
(I, Q, U, V, 1) evolves under the 5 x 5 matrix [[-K, j], [0, 0]] with K the
simplified transfer matrix (alpha_I on the diagonal, rho_V coupling Q and U),
and the step is its matrix exponential (scipy.linalg.expm). The two agree to
FP64 rounding (tests/test_stokes_oracle.py), which pins the restatement
without a GPU; the reference's own known answers
(tests/cuda_stokes_test.cu:170-330: pure rotation, pure absorption, the
polarization bound, a rotation round trip, zero input) pin both.
"""
from __future__ import annotations

import numpy as np


def stokes_step(s, jI, jQ, jU, jV, alpha, rho, ds):
    """One step from Stokes state s = (I, Q, U, V); returns the new state
    (src/cuda/device_physics.cuh:2216-2284)."""
    i, q, u, v = (float(x) for x in s)
    if ds <= 0.0:
        return np.array([i, q, u, v])
    A = max(alpha, 0.0)
    R = rho
    tau = A * ds
    E = np.exp(-tau) if tau < 700.0 else 0.0
    phi = R * ds
    c, sn = np.cos(phi), np.sin(phi)

    def scalar(x, j):  # :2231-2249
        if A < 1e-30:
            return x + j * ds
        if tau < 1e-4:
            return x * (1.0 - tau) + j * ds
        return x * E + (j / A) * (1.0 - E)

    i_new, v_new = scalar(i, jI), scalar(v, jV)
    q_hom = E * (q * c - u * sn)
    u_hom = E * (q * sn + u * c)
    D = A * A + R * R
    if D < 1e-60:  # :2259-2262 pure emission
        q_new, u_new = q + jQ * ds, u + jU * ds
    elif A < 1e-15 * abs(R):  # :2263-2268 rotation only
        ic, is_ = sn / R, (1.0 - c) / R
        q_new, u_new = jQ * ic - jU * is_ + q_hom, jQ * is_ + jU * ic + u_hom
    elif abs(R) < 1e-15 * A:  # :2269-2273 absorption only
        w = ds - 0.5 * tau * ds if tau < 1e-4 else (1.0 - E) / A
        q_new, u_new = jQ * w + q_hom, jU * w + u_hom
    else:  # :2274-2280
        ec, es = E * c, E * sn
        ic = (A * (1.0 - ec) + R * es) / D
        is_ = (R * (1.0 - ec) - A * es) / D
        q_new, u_new = jQ * ic - jU * is_ + q_hom, jQ * is_ + jU * ic + u_hom
    return np.array([i_new, q_new, u_new, v_new])


def stokes_step_expm(s, jI, jQ, jU, jV, alpha, rho, ds):
    """The same step as the exponential of the augmented transfer matrix."""
    from scipy.linalg import expm

    if ds <= 0.0:
        return np.asarray(s, dtype=np.float64).copy()
    A = max(alpha, 0.0)
    M = np.zeros((5, 5))
    M[0, 0] = M[1, 1] = M[2, 2] = M[3, 3] = -A
    M[1, 2] = -rho  # dQ/ds = ... - rho U
    M[2, 1] = rho   # dU/ds = ... + rho Q
    M[:4, 4] = (jI, jQ, jU, jV)
    x = np.append(np.asarray(s, dtype=np.float64), 1.0)
    return (expm(M * ds) @ x)[:4]
