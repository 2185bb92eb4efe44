"""include/bh_physics_compat.hpp: the reference's scalar C++ Kerr API
(physics::kerrPotentials, kerrStepMino, KerrRaytracer::trace / traceEquatorial,
src/physics/kerr.h:362-453, raytracer.h:46-399) over the C ABI.

A C++23 program (tests/cpp/physics_compat_main.cpp) written the way a
reference caller is written is compiled against the header and linked with
libblackhole_b200.so only. On the CPU: it compiles, links and its pure
helpers return the reference's values. On the GPU: its kerrPotentials,
kerrStepMino and KerrRaytracer results equal the golden vectors of the
reference's own compiled kerr.cpp, at the tolerances of the batched API's
parity tests (CUDA's sin/cos against glibc's), and a trace with the path
recorded ends where the batched trace ends.
"""
from __future__ import annotations

import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import load_golden
from test_oracle_pins import trace_case

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "physics_compat_main.cpp"
STATE = ("r", "theta", "phi", "t", "sign_r", "sign_theta")


@pytest.fixture(scope="module")
def program(tmp_path_factory, lib):
    exe = tmp_path_factory.mktemp("physics_compat") / "physics_compat_main"
    libdir = ROOT / "blackhole_b200" / "lib"
    cmd = ["g++", "-std=c++23", "-O2", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}", str(SRC),
           f"-L{libdir}", "-lblackhole_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def run(program, mode, arr, tmp_path):
    inp, out = tmp_path / f"{mode}.in", tmp_path / f"{mode}.out"
    np.ascontiguousarray(arr, np.float64).tofile(inp)
    r = subprocess.run([str(program), mode, str(inp), str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return np.fromfile(out, np.float64)


def test_compat_header_compiles_links_and_helpers_match(program):
    r = subprocess.run([str(program), "info"], capture_output=True, text=True, check=True)
    e, lz, q, theta, sign_r, sign_theta = map(float, r.stdout.split())
    # kerrEquatorialConsts(5, 2) and kerrEquatorialState(30, 0.25, -0.5) (kerr.h:396-437)
    assert (e, lz, q) == (2.0, 10.0, 0.0)
    assert theta == 0.5 * math.pi and sign_r == -1.0 and sign_theta == 1.0


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["geom", "cgs"])
def test_compat_potentials_and_step_match_reference(cuda, program, tag, tmp_path):
    g = load_golden("kerr_step_ref.npz")
    n = len(g[f"{tag}_e"])
    cols = [g[f"{tag}_in_{k}"] for k in STATE] + [g[f"{tag}_{k}"] for k in ("e", "lz", "q", "dlam")]
    arr = np.concatenate([[n, float(g[f"{tag}_mass"]), float(g[f"{tag}_a"])], np.concatenate(cols)])
    pot = run(program, "potentials", arr, tmp_path).reshape(n, 4)
    for j, k in enumerate(("r_pot", "dr_pot", "theta_pot", "dtheta_pot")):
        ref = g[f"{tag}_pot_{k}"]
        scale = np.maximum(np.abs(ref) + 1e-300, np.abs(ref).max() * 1e-6)
        assert np.all(np.abs(pot[:, j] - ref) <= 1e-12 * scale), k
    step = run(program, "step", arr, tmp_path).reshape(n, 6)
    for j, k in enumerate(STATE[:4]):
        np.testing.assert_allclose(step[:, j], g[f"{tag}_step1_{k}"], rtol=1e-13, atol=1e-300, err_msg=k)
    np.testing.assert_array_equal(step[:, 4], g[f"{tag}_step1_sign_r"])


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["geom_a0", "geom_a09"])
def test_compat_raytracer_matches_reference(cuda, program, tag, tmp_path):
    g = load_golden("kerr_trace_ref.npz")
    (mass, a, _r_h, r_esc, step, max_steps), eq, gen = trace_case(g, tag)
    for kind, (st, e, lz, q) in (("eq", eq), ("gen", gen)):
        n = len(e)
        cols = [st[k] for k in STATE] + [e, lz, q]
        arr = np.concatenate([[n, mass, a, step, max_steps, r_esc], np.concatenate(cols)])
        out = run(program, "trace", arr, tmp_path)
        res, one = out[: 7 * n].reshape(n, 7), out[7 * n:]
        status, steps = res[:, 0].astype(int), res[:, 1].astype(int)
        np.testing.assert_array_equal(status, g[f"{tag}_{kind}_status"], err_msg=f"{kind} status")
        assert np.all(np.abs(steps - g[f"{tag}_{kind}_steps"]) <= 1), kind
        same = steps == g[f"{tag}_{kind}_steps"]
        for j, k in ((3, "r"), (4, "theta"), (5, "phi")):
            np.testing.assert_allclose(res[same, j], g[f"{tag}_{kind}_{k}"][same], rtol=1e-7, err_msg=f"{kind} {k}")
        # element 0 again, one kerrPotentials / kerrStepMino round trip per step, with its path recorded
        assert one[0] == res[0, 0] and one[1] == res[0, 1], (one[:2], res[0, :2])
        np.testing.assert_allclose(one[2:7], res[0, 2:7], rtol=1e-12, atol=1e-300)
        assert one[7] == one[1] + 1  # the start point and one point per step
