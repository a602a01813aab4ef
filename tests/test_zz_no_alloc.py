"""rt_render_device_noalloc: the render entry point for hosts that cannot
allocate device memory while rendering (a device-memory budget fixed at
start-up, or a latency-critical render thread where the device-synchronising
cudaMalloc/cudaFree are not allowed). Its scratch lives in one fixed array in
the library; this test checks, through the C-ABI, that two calls in a row give
the same film as the allocating rt_render_device, and that an oversized
window and a wavefront request are refused. Collected last so that a run
stopping at the first failure has already run every other test."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import rt

pytestmark = pytest.mark.gpu

abi = rt.abi


def test_noalloc_matches_allocating_render_twice(cornell_world):
    import torch
    lib = abi.load()
    pw = abi.PackedWorld(cornell_world)
    h = C.c_void_p()
    abi.check(lib.rt_scene_create(pw.ref(), C.byref(h)), "rt_scene_create")
    try:
        W, H = 96, 64
        p = abi.render_params(W, H, 64, 8, kernel=abi.KERNEL_MEGAKERNEL)
        ref = torch.zeros((3, H, W), dtype=torch.float32, device="cuda")
        st = abi.RtStats()
        abi.check(lib.rt_render_device(h, C.byref(p), C.c_void_p(ref.data_ptr()), C.byref(st)), "rt_render_device")
        expect = ref.cpu().numpy()
        assert np.all(np.isfinite(expect)) and expect.mean() > 0
        for call in range(2):
            film = torch.full((3, H, W), -1.0, dtype=torch.float32, device="cuda")
            st2 = abi.RtStats()
            abi.check(lib.rt_render_device_noalloc(h, C.byref(p), C.c_void_p(film.data_ptr()), C.byref(st2)),
                      f"rt_render_device_noalloc call {call}")
            assert st2.samples == W * H * 64
            np.testing.assert_allclose(film.cpu().numpy(), expect, rtol=1e-4, atol=1e-6)
        # a window: only its pixels are written, the rest of the film is zeroed
        pw_ = abi.render_params(W, H, 64, 8, kernel=abi.KERNEL_MEGAKERNEL, pixel_x0=16, pixel_y0=8, window_w=32,
                                window_h=16)
        film = torch.full((3, H, W), -1.0, dtype=torch.float32, device="cuda")
        abi.check(lib.rt_render_device_noalloc(h, C.byref(pw_), C.c_void_p(film.data_ptr()), C.byref(st2)))
        f = film.cpu().numpy()
        np.testing.assert_allclose(f[:, 8:24, 16:48], expect[:, 8:24, 16:48], rtol=1e-4, atol=1e-6)
        assert np.all(f[:, :8] == 0)
        # beyond the fixed maximum: refused with a clear error, nothing launched
        big = abi.render_params(4096, 4096, 1, 1, kernel=abi.KERNEL_MEGAKERNEL)
        rc = lib.rt_render_device_noalloc(h, C.byref(big), C.c_void_p(ref.data_ptr()), C.byref(st2))
        assert rc == -1 and b"allocation-free maximum" in lib.rt_last_error()
        # the wavefront's queues need allocated memory: a wavefront request is
        # refused, not silently rendered by the megakernel
        wf = abi.render_params(W, H, 64, 8, kernel=abi.KERNEL_WAVEFRONT)
        rc = lib.rt_render_device_noalloc(h, C.byref(wf), C.c_void_p(ref.data_ptr()), C.byref(st2))
        assert rc == -1 and b"megakernel" in lib.rt_last_error()
    finally:
        lib.rt_scene_destroy(h)
