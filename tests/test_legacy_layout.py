"""The legacy launch ABI (include/bh_legacy.h) on the CPU: BH_LaunchParams has
the reference's byte layout (size and every field offset, recorded from the
reference's own header by tests/golden/make_launch_params_layout.py: the check
tests/cuda_kernel_launch_test.cpp:32-104 makes, against the current header),
the variant enum keeps its values, and the calls reject bad arguments
before touching a GPU."""
from __future__ import annotations

import ctypes as C
import json
import subprocess

import numpy as np
import pytest

from conftest import ROOT

LAYOUT = json.loads((ROOT / "tests" / "golden" / "launch_params_layout.json").read_text())


def _compile_and_run(tmp_path, body: str) -> str:
    src = tmp_path / "t.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "bh_legacy.h"\nint main(void) {\n'
                   + body + "  return 0;\n}\n")
    exe = tmp_path / "t"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    return subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout


def test_launch_params_layout_matches_reference(tmp_path):
    names = LAYOUT["fields"]
    body = '  printf("size %zu\\n", sizeof(struct BH_LaunchParams));\n'
    body += "".join(f'  printf("{n} %zu\\n", offsetof(struct BH_LaunchParams, {n}));\n' for n in names)
    got = dict(line.split() for line in _compile_and_run(tmp_path, body).splitlines())
    assert int(got.pop("size")) == LAYOUT["size"]
    assert {k: int(v) for k, v in got.items()} == LAYOUT["offsets"]


def test_kernel_variant_values(tmp_path):
    out = _compile_and_run(tmp_path, '  printf("%d %d %d %d %d\\n", BH_KERNEL_FP32_BASELINE, BH_KERNEL_FP32_COARSENED,'
                                     ' BH_KERNEL_FP16_STORAGE, BH_KERNEL_FP16_H2_ILP, BH_KERNEL_COUNT);\n')
    assert out.split() == ["0", "1", "2", "3", "4"]


def test_launch_params_mirror(lib):
    from blackhole_b200 import legacy

    assert C.sizeof(legacy.LaunchParams) == LAYOUT["size"]
    for name, off in LAYOUT["offsets"].items():
        assert getattr(legacy.LaunchParams, name).offset == off, name


def test_rejects_bad_arguments_without_gpu(lib):
    from blackhole_b200 import legacy

    p = legacy.bridge_params(0.9, 30.0, 1.2, 1.0, 64, 64)
    assert lib.bh_launch_geodesic_kernel(None, C.byref(p), 0, None) == -1
    assert b"framebuffer" in lib.bh_last_error()
    bad = legacy.bridge_params(0.9, 30.0, 1.2, 1.0, 0, 64)
    assert lib.bh_launch_geodesic_kernel(C.c_void_p(16), C.byref(bad), 0, None) == -1
    bad = legacy.bridge_params(1.5, 30.0, 1.2, 1.0, 64, 64)
    assert lib.bh_launch_geodesic_kernel(C.c_void_p(16), C.byref(bad), 0, None) == -1
    assert lib.bh_launch_geodesic_kernel(C.c_void_p(16), C.byref(p), 7, None) == -1
    assert lib.bh_select_kernel_variant() == 0
    assert lib.bhbHasCuda() == 1
    out = np.zeros(4, np.float32)
    assert lib.bhbCudaRenderRaytraced(C.c_float(0.9), C.c_float(30.0), C.c_float(1.2), 0, 1,
                                      out.ctypes.data_as(C.c_void_p)) == -1
    assert lib.bhbCudaTraceGeodesics(C.c_double(0.9), C.c_double(100.0), C.c_double(1.0), C.c_double(-5),
                                     C.c_double(5), 2, C.c_double(-5), C.c_double(5), 2, 0, C.c_double(0.1),
                                     None, None) == -1
    assert lib.bhCudaRegisterLut(None, 0, 1, 0) == -1
    lib.bhCudaShutdown(None)


@pytest.mark.parametrize("incl", [0.0, 1.2, np.pi / 2])
def test_bridge_camera_basis_is_orthonormal_and_looks_at_the_hole(lib, incl):
    from blackhole_b200 import legacy

    p = legacy.bridge_params(0.5, 40.0, incl, 1.0, 32, 16)
    B = np.array(p.cam_basis, np.float64).reshape(3, 3).T  # columns right, up, forward
    assert np.allclose(B.T @ B, np.eye(3), atol=1e-6)
    pos = np.array(p.cam_pos, np.float64)
    assert np.allclose(B[:, 2], -pos / np.linalg.norm(pos), atol=1e-6)
    assert np.isclose(np.linalg.norm(pos), 40.0)


def test_postprocess_restatement_properties():
    """The post-processing restatement (oracle/legacy_oracle.py) on cases with
    a closed form: a constant frame blurs to itself, so the composite adds
    4 x strength x its bright-pass; above every pixel's luminance the bloom
    is nothing; the tone map of 0 is 0 and saturates at 1."""
    from oracle import legacy_oracle as LO

    h, w = 9, 13
    c = np.array([2.0, 1.0, 0.5], np.float32)
    fb = np.broadcast_to(np.append(c, 0.25), (h, w, 4)).astype(np.float32)
    lum = 0.2126 * 2.0 + 0.7152 * 1.0 + 0.0722 * 0.5
    bright = c.astype(np.float64) * (lum - 0.4) / lum
    composite = np.concatenate([np.broadcast_to(c + 0.5 * 4 * bright, (h, w, 3)), np.ones((h, w, 1))], -1)
    plain = LO.postprocess(composite, 1e9, 0.0, 2.0)
    np.testing.assert_allclose(LO.postprocess(fb, 0.4, 0.5, 2.0), plain, rtol=1e-12)
    rng = np.random.default_rng(3)
    x = rng.random((h, w, 4)).astype(np.float32)
    np.testing.assert_array_equal(LO.postprocess(x, 10.0, 3.0, 1.5), LO.postprocess(x, 10.0, 0.0, 1.5))
    out = LO.postprocess(np.zeros((h, w, 4), np.float32), 1.0, 1.0, 12.0)
    assert np.all(out[..., :3] == 0.0) and np.all(out[..., 3] == 1.0)
    out = LO.postprocess(np.full((h, w, 4), 1e6, np.float32), 1.0, 0.0, 12.0)
    np.testing.assert_allclose(out[..., :3], 1.0)
