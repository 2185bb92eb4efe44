"""bh_kerr_trace_image_host_noalloc: the image trace for callers that cannot
allocate device memory (a plug-in whose host application owns the GPU memory
pool or forbids cudaMalloc on its render thread, a real-time loop that must
not block on an allocation).

The entry point takes host output buffers like bh_kerr_trace_image_host but
stages everything in one fixed device array instead of allocating. These
tests call it through the C ABI and compare it with the allocating entry
point bit for bit (the tolerance of every FP64 image test here), twice in a
row, so the second call also shows that the reused scratch is cleared. The
file is named to be collected last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("cls", "steps", "n_cross", "r_hit", "phi_hit", "g", "flux", "intensity", "theta_inf", "phi_inf")


def host_arrays(scene, fields=FIELDS):
    n = scene.width * scene.height
    mc = scene.max_crossings
    out = {}
    for k in fields:
        shape = (mc, n) if k in ("r_hit", "phi_hit", "g") else (n,)
        out[k] = np.full(shape, -7, np.int32 if k in ("cls", "steps", "n_cross") else np.float64)
    return out


def struct_for(arrs):
    from blackhole_b200 import _abi

    o = _abi.KerrImageOut()
    for k, v in arrs.items():
        setattr(o, k, v.ctypes.data)
    return o


def call(lib, fn_name, scene, arrs, *extra):
    from blackhole_b200 import _abi

    rc = getattr(lib, fn_name)(C.byref(scene), C.byref(struct_for(arrs)), *extra)
    if rc != 0:
        raise RuntimeError(lib.bh_last_error().decode())
    return arrs


@pytest.mark.parametrize("integrator,max_cross,w,h", [(1, 3, 96, 80), (0, 1, 64, 64)])
def test_noalloc_matches_allocating_entry_point_twice(cuda, lib, integrator, max_cross, w, h):
    from blackhole_b200 import _abi

    s = _abi.default_scene(width=w, height=h, integrator=integrator, max_crossings=max_cross)
    ref = call(lib, "bh_kerr_trace_image_host", s, host_arrays(s))
    for attempt in range(2):
        got = call(lib, "bh_kerr_trace_image_host_noalloc", s, host_arrays(s), None)
        for k in FIELDS:
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"{k} (call {attempt + 1})")


@pytest.mark.parametrize("integrator", [1, 2])
def test_noalloc_calls_allocate_no_device_memory(cuda, lib, integrator):
    """The library counts every device allocation it makes
    (bh_debug_device_allocations): neither a first nor a second call of the
    no-allocation entry point adds one, with a stepping or the closed-form
    integrator (whose fallback list also lives in the fixed array). The
    device's free memory, a secondary check that other processes can
    disturb, stays the same across the second call."""
    import torch

    from blackhole_b200 import _abi

    s = _abi.default_scene(width=80, height=72, integrator=integrator, max_crossings=2)
    before = lib.bh_debug_device_allocations()
    call(lib, "bh_kerr_trace_image_host_noalloc", s, host_arrays(s), None)
    assert lib.bh_debug_device_allocations() == before
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    got = call(lib, "bh_kerr_trace_image_host_noalloc", s, host_arrays(s), None)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert lib.bh_debug_device_allocations() == before
    assert free_after == free_before
    assert (got["cls"] >= 0).all()


def test_noalloc_on_a_caller_stream(cuda, lib):
    import torch

    from blackhole_b200 import _abi

    s = _abi.default_scene(width=40, height=36, integrator=1, max_crossings=3)
    ref = call(lib, "bh_kerr_trace_image_host", s, host_arrays(s))
    st = torch.cuda.Stream()
    got = call(lib, "bh_kerr_trace_image_host_noalloc", s, host_arrays(s), C.c_void_p(st.cuda_stream))
    for k in FIELDS:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


def test_noalloc_rejects_images_beyond_its_scratch(cuda, lib):
    from blackhole_b200 import _abi

    s = _abi.default_scene(width=1024, height=1024)  # ~71 MB of outputs > 32 MiB
    arrs = host_arrays(s)
    rc = lib.bh_kerr_trace_image_host_noalloc(C.byref(s), C.byref(struct_for(arrs)), None)
    assert rc == -1
    msg = lib.bh_last_error().decode()
    assert "bh_kerr_trace_image_host_noalloc" in msg and "scratch" in msg
    assert (arrs["cls"] == -7).all()  # nothing written
    # fewer requested fields fit: cls + g of the same image is 12 MB
    small = host_arrays(s, fields=("cls", "g"))
    call(lib, "bh_kerr_trace_image_host_noalloc", _abi.default_scene(width=1024, height=1024, max_steps=0), small,
         None)
    assert (small["cls"] == 3).all()
