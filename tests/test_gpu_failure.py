"""Failure detection without a GPU fault.

The reference's contract on a failure is an error return, after which its
caller re-initialises the backend (src/cuda/cuda_render_manager.h:155-199).
Here the failures are made on purpose and checked end to end, on one GPU:

* bounded device waits: the network's tensor-core kernels (fused inference
  and the training GEMMs) wait on mbarriers for other warps' progress, each
  wait bounded by a host-settable limit. At a limit of 1 ns every wait that is
  not already satisfied runs out: the kernel records an error code, lets the
  loads and MMAs its own threads started land, frees its tensor memory and
  returns. The C call reports -1 (host-buffer render) or the code
  (bh_surrogate_device_error), and the next call at the default limit gives
  the same result as before the failure;
* host allocations: bh_debug_fail_device_allocation makes the library's n-th
  device allocation from now fail as if the device were out of memory. The
  entry point returns -1 with a message naming the allocation, keeps its
  cached buffers consistent, and the next call succeeds with the same
  outputs.

Nothing here faults, traps or hangs a GPU: every failure is a status that
the host reads.
"""
from __future__ import annotations

import math
import threading

import numpy as np
import pytest
import torch

from blackhole_b200 import _abi, kerr
from blackhole_b200 import surrogate as S

pytestmark = pytest.mark.gpu


def c4_scene(W, **kw):
    args = dict(width=W, height=W, spin=0.9, theta_obs=math.radians(60), integrator=1, max_crossings=1, precision=1)
    args.update(kw)
    return kerr.scene(**args)


def rand_inputs(n, seed):
    g = torch.Generator().manual_seed(seed)
    u = torch.rand(n, 4, generator=g, dtype=torch.float64)
    x = torch.stack([-15 + 30 * u[:, 0], -15 + 30 * u[:, 1], 0.998 * u[:, 2],
                     torch.cos(torch.deg2rad(5 + 84 * u[:, 3]))], 1)
    return x.float()


def test_surrogate_waits_run_out_and_the_next_call_is_correct(cuda):
    net = S.Surrogate(max_batch=256, seed=3)
    s = c4_scene(128)
    ref = net.trace_image_host(s)
    x = rand_inputs(1000, 5).cuda()
    head_ref = net.forward(x).clone()
    assert net.device_error() == 0

    net.set_wait_limit(1)
    with pytest.raises(RuntimeError, match="bounded device wait"):
        net.trace_image_host(s)
    assert net.device_error() == 0  # the host call read and cleared the code it reported
    net.forward(x)
    assert net.device_error() != 0  # asynchronous call: the code waits for the host to read it
    assert net.device_error() == 0

    net.set_wait_limit(0)
    got = net.trace_image_host(s)
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    assert torch.equal(net.forward(x), head_ref)
    assert net.device_error() == 0


def test_training_gemm_waits_run_out_and_recover(cuda):
    net = S.Surrogate(max_batch=512, seed=7)
    x = rand_inputs(512, 3).cuda()
    rng = np.random.default_rng(4)
    t = np.zeros((512, 16), np.float32)
    t[:, 0] = rng.integers(0, 3, 512)
    t[:, 2:12] = rng.normal(0.0, 0.5, (512, 10))
    t = torch.from_numpy(t).cuda()
    g_ref, _ = net.gradients(x, t)
    g_ref = g_ref.clone()
    assert net.device_error() == 0
    net.set_wait_limit(1)
    net.gradients(x, t)
    assert net.device_error() != 0
    net.set_wait_limit(0)
    g, _ = net.gradients(x, t)
    assert net.device_error() == 0
    torch.testing.assert_close(g, g_ref, rtol=1e-5, atol=1e-7)


def _in_new_thread(fn):
    """Run fn on a fresh host thread (the host-buffer entry points keep their
    staging buffers per thread, so its first call must allocate)."""
    box = {}

    def run():
        try:
            box["value"] = fn()
        except BaseException as e:  # re-raised on the caller's thread
            box["error"] = e

    th = threading.Thread(target=run)
    th.start()
    th.join()
    if "error" in box:
        raise box["error"]
    return box["value"]


def test_image_host_entry_reports_a_failed_allocation(cuda, lib):
    s = _abi.default_scene(width=64, height=48, integrator=1, max_crossings=2)
    ref = kerr.trace_image_host(s)

    def body():
        before = lib.bh_debug_device_allocations()
        assert lib.bh_debug_fail_device_allocation(1) == 0
        try:
            kerr.trace_image_host(s)
            raise AssertionError("the injected allocation failure was not reported")
        except RuntimeError as e:
            msg = str(e)
        got = kerr.trace_image_host(s)
        return msg, got, lib.bh_debug_device_allocations() - before

    msg, got, new_allocs = _in_new_thread(body)
    assert "cudaMalloc(output buffers)" in msg and "out of memory" in msg, msg
    assert new_allocs == 1  # the retry allocated once; the failed attempt allocated nothing
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


def test_surrogate_reports_failed_allocations_at_every_stage(cuda, lib):
    """A fresh network's first host-buffer render allocates its output
    staging, then the renderer's buffers: failing the 1st, 3rd and 6th of
    those in turn leaves each partly built state consistent, and the render
    after them equals a render that never failed. Creating a network reports
    a failed allocation the same way."""
    s = c4_scene(96)
    ref = S.Surrogate(max_batch=128, seed=3).trace_image_host(s)
    net = S.Surrogate(max_batch=128, seed=3)
    for nth in (1, 3, 6):
        assert lib.bh_debug_fail_device_allocation(nth) == 0
        with pytest.raises(RuntimeError, match="out of memory"):
            net.trace_image_host(s)
    assert lib.bh_debug_fail_device_allocation(0) == 0
    got = net.trace_image_host(s)
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    assert lib.bh_debug_fail_device_allocation(5) == 0
    with pytest.raises(RuntimeError, match="out of memory"):
        S.Surrogate(max_batch=128, seed=1)
    assert lib.bh_debug_fail_device_allocation(0) == 0
    S.Surrogate(max_batch=128, seed=1).close()
