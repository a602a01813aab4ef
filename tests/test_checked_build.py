"""The checked build (lib/librt3d_checked.so, compiled with -DRT_CHECKED): every
index a kernel takes from scene data or from the wavefront's queues is tested
against its array's length, and an index out of range makes the call return
RT_ERR_BOUNDS instead of reading outside the array. It stands in for
compute-sanitizer's memcheck, which is not available on the GPU hosts.

CPU: the checked library loads, exports every symbol of include/rt3d.h and
says it is the checked build. GPU: the main paths (both kernels with every ray
order and node layout, the glass walk and the medium, traces, capture, the
adjoint, a batch) run clean under it and give the product build's results.
The whole GPU suite can also be run against it: RT3D_LIB=<path> pytest -m gpu.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from conftest import camera_rays, rt
from test_abi import declared_functions

abi = rt.abi

needs_checked = pytest.mark.skipif(not os.path.exists(abi.CHECKED_LIB_PATH),
                                   reason="the checked build is not built")


@needs_checked
def test_checked_library_exports_the_abi():
    lib = abi.load(abi.CHECKED_LIB_PATH)
    for n in declared_functions():
        assert hasattr(lib, n), n
    assert lib.rt_checked_build() == 1
    assert lib.rt_abi_version() == abi.load().rt_abi_version()


def test_product_library_is_not_the_checked_build():
    if os.environ.get("RT3D_LIB"):
        pytest.skip("RT3D_LIB selects another build")
    assert abi.load().rt_checked_build() == 0


class _Scene:
    def __init__(self, lib, world):
        self.lib = lib
        self.packed = abi.PackedWorld(world)
        h = C.c_void_p()
        abi.check(lib.rt_scene_create(self.packed.ref(), C.byref(h)), "rt_scene_create")
        self.h = h

    def render(self, p):
        out = np.zeros((3, p.height, p.width), np.float32)
        st = abi.RtStats()
        rc = self.lib.rt_render(self.h, C.byref(p), abi.ptr(out), C.byref(st))
        assert rc == 0, (rc, self.lib.rt_last_error())
        return out

    def close(self):
        self.lib.rt_scene_destroy(self.h)


def _both(world):
    return _Scene(abi.load(), world), _Scene(abi.load(abi.CHECKED_LIB_PATH), world)


WF = abi.KERNEL_WAVEFRONT
MK = abi.KERNEL_MEGAKERNEL


@needs_checked
@pytest.mark.gpu
@pytest.mark.parametrize("which", ["cornell", "icospheres", "volume", "spheres", "smooth"])
def test_checked_build_renders_clean_and_equal(which):
    world = {"cornell": lambda: rt.scenes.cornell(), "icospheres": lambda: rt.scenes.throughput_scene(8, 3),
             "volume": lambda: rt.scenes.cornell_volume(density=0.3), "spheres": lambda: rt.scenes.cornell_spheres(),
             "smooth": lambda: rt.scenes.cornell_smooth()}[which]()
    prod, chk = _both(world)
    try:
        runs = [dict(kernel=MK)]
        for g in (1, 2, 3, 4):
            runs.append(dict(kernel=WF, wavefront_size=1 << 14, ray_groups=g))
        runs += [dict(kernel=WF, wavefront_size=1 << 14, node_layout=4),
                 dict(kernel=WF, wavefront_size=1 << 14, ray_fetch=2, ray_groups=1),
                 dict(kernel=WF, wavefront_size=1 << 14, sort_materials=0)]
        for kw in runs:
            p = abi.render_params(40, 32, 32, 12, **kw)
            a, b = prod.render(p), chk.render(p)
            np.testing.assert_allclose(b, a, rtol=1e-4, atol=1e-6, err_msg=str(kw))
        rays = camera_rays(world, 64, 64)
        for layout in (2, 4):
            ha, hb = np.zeros((rays.shape[0], 6), np.int32), np.zeros((rays.shape[0], 6), np.int32)
            abi.check(prod.lib.rt_trace_closest(prod.h, abi.ptr(rays), rays.shape[0], 1e-4, 3.4e38, abi.ptr(ha),
                                                layout))
            abi.check(chk.lib.rt_trace_closest(chk.h, abi.ptr(rays), rays.shape[0], 1e-4, 3.4e38, abi.ptr(hb),
                                               layout), "checked rt_trace_closest")
            assert np.array_equal(ha, hb)
    finally:
        prod.close()
        chk.close()


@needs_checked
@pytest.mark.gpu
def test_checked_build_capture_adjoint_and_batch_run_clean():
    lib = abi.load(abi.CHECKED_LIB_PATH)
    world = rt.scenes.cornell_sphere(dict(sheen=0.5))
    s = _Scene(lib, world)
    try:
        p = abi.render_params(24, 24, 16, 8)
        beauty = np.zeros((3, 24, 24), np.float32)
        planes = {k: np.zeros((3, 24, 24), np.float32) for k in ("beauty_a", "beauty_b", "albedo_a", "albedo_b",
                                                                  "normal_a", "normal_b")}
        planes.update({k: np.zeros((24, 24), np.float32) for k in ("depth_a", "depth_b")})
        cap = abi.RtCapture(**{k: v.ctypes.data for k, v in planes.items()})
        st = abi.RtStats()
        abi.check(lib.rt_render_capture(s.h, C.byref(p), abi.ptr(beauty), C.byref(cap), C.byref(st)),
                  "checked rt_render_capture")
        n = len(world.materials) * abi.ADJ_PER_MATERIAL + abi.ADJ_GLOBAL
        grad = np.zeros(n, np.float32)
        dimg = np.ones((3, 24, 24), np.float32)
        abi.check(lib.rt_adjoint(s.h, C.byref(p), abi.ptr(dimg), None, abi.ptr(grad), n, C.byref(st)),
                  "checked rt_adjoint")
        assert np.all(np.isfinite(grad)) and np.any(grad != 0)
        reqs = (abi.RtRequest * 3)()
        outs = [np.zeros((3, r, r), np.float32) for r in (16, 24, 8)]
        for i, r in enumerate((16, 24, 8)):
            reqs[i].scene, reqs[i].width, reqs[i].height, reqs[i].spp, reqs[i].max_depth = 0, r, r, 8, 6
            reqs[i].camera = abi.camera_desc(world.camera)
        scenes = (C.c_void_p * 1)(s.h)
        optrs = (C.c_void_p * 3)(*[o.ctypes.data for o in outs])
        common = abi.render_params(1, 1, 1, 1, kernel=WF, wavefront_size=1 << 12)
        abi.check(lib.rt_render_batch(scenes, 1, reqs, 3, C.byref(common), optrs, C.byref(st)), "checked batch")
        assert all(np.all(np.isfinite(o)) for o in outs)
    finally:
        s.close()
