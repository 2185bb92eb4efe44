"""CPU checks of the C ABI: the library loads, exports every function that
include/*.h declares, and its host-only entry points (defaults, validation,
KerrRaytracer parameters) behave; no call here touches a GPU."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, load_golden

HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions(path: Path) -> list[str]:
    text = path.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    text = re.sub(r"^\s*#[^\n]*", "", text, flags=re.M)
    text = re.sub(r"typedef\s+struct\s*\w*\s*\{.*?\}\s*\w+\s*;", "", text, flags=re.S)
    text = re.sub(r"(struct|enum)\s+\w+\s*\{.*?\}\s*;", "", text, flags=re.S)
    names = re.findall(r"\b([a-zA-Z_]\w*)\s*\([^;{}]*\)\s*;", text)
    return sorted(set(n for n in names if n not in ("if", "while", "sizeof")))


def test_headers_declare_functions():
    assert HEADERS, "include/ has no headers"
    for h in HEADERS:
        assert declared_functions(h), h


def test_library_exports_every_declared_symbol(lib):
    missing = []
    for h in HEADERS:
        for name in declared_functions(h):
            if not hasattr(lib, name):
                missing.append(f"{h.name}:{name}")
    assert not missing, missing


def test_headers_compile_as_c99(tmp_path):
    import subprocess

    src = tmp_path / "t.c"
    src.write_text("".join(f'#include "{h}"\n' for h in HEADERS) + "int main(void){return 0;}\n")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-pedantic", "-c", str(src), "-o",
                    str(tmp_path / "t.o")], check=True)


def test_abi_struct_layout(lib, tmp_path):
    """ctypes mirrors match the C compiler's size and every field offset (the
    check tests/cuda_kernel_launch_test.cpp:32-104 makes for BH_LaunchParams)."""
    import subprocess

    from blackhole_b200 import _abi

    assert lib.bh_abi_version() == 1
    structs = {"BH_KerrScene": _abi.KerrScene, "BH_KerrImageOut": _abi.KerrImageOut,
               "BH_KerrRaytracerParams": _abi.KerrRaytracerParams, "BH_KerrStateSoA": _abi.KerrStateSoA,
               "BH_KerrConstsSoA": _abi.KerrConstsSoA}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{ROOT / "include" / "bh_kerr.h"}"',
             "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                       text=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, f"{cname}.{f}"


def test_scene_defaults_and_validation(lib):
    from blackhole_b200 import _abi

    s = _abi.KerrScene()
    lib.bh_kerr_scene_defaults(C.byref(s))
    assert (s.width, s.height, s.max_steps) == (256, 256, 20000)
    assert s.spin == 0.9 and s.r_obs == 1000.0 and abs(s.theta_obs - np.pi / 3) < 1e-15
    assert lib.bh_kerr_scene_validate(C.byref(s)) == 0
    for field, value in (("spin", 1.0), ("theta_obs", 3.2), ("max_crossings", 0), ("step_coeff", 0.0),
                         ("precision", 5), ("potential_form", 2), ("alpha_max", -20.0)):
        bad = _abi.KerrScene.from_buffer_copy(s)
        setattr(bad, field, value)
        assert lib.bh_kerr_scene_validate(C.byref(bad)) == -1, field
        assert lib.bh_last_error().decode()


def test_trace_image_rejects_invalid_scene_without_gpu(lib):
    from blackhole_b200 import _abi

    s = _abi.default_scene(spin=2.0)
    o = _abi.KerrImageOut()
    assert lib.bh_kerr_trace_image(C.byref(s), C.byref(o), None) == -1
    assert b"spin" in lib.bh_last_error()


def test_set_launch_validation(lib):
    assert lib.bh_kerr_set_launch(33, 0) == -1
    assert lib.bh_kerr_set_launch(256, 0) == -1
    assert lib.bh_kerr_set_launch(64, 2) == 0
    assert lib.bh_kerr_set_launch(0, 0) == 0


def test_raytracer_defaults_match_reference(lib):
    from blackhole_b200 import _abi

    g = load_golden("kerr_trace_ref.npz")
    for tag in ("cgs_a0", "cgs_a09"):
        p = _abi.KerrRaytracerParams()
        assert lib.bh_kerr_raytracer_defaults(float(g[f"{tag}_mass"]), float(g[f"{tag}_a"]), C.byref(p)) == 0
        assert p.r_horizon == float(g[f"{tag}_r_horizon"])
        assert p.r_escape == float(g[f"{tag}_r_escape"])
        assert p.step_size == float(g[f"{tag}_step_size"])
        assert p.max_steps == 10000


def test_raytracer_clamps_overextremal_spin_like_physics_kerr(lib):
    from blackhole_b200 import _abi

    mass = 1.98841e33
    m = 6.67430e-8 * mass / 2.99792458e10**2
    p = _abi.KerrRaytracerParams()
    lib.bh_kerr_raytracer_defaults(mass, 1.5 * m, C.byref(p))
    assert p.a == pytest.approx(0.998 * m, rel=1e-15)
