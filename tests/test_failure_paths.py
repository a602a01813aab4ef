"""Failure paths of the C-ABI, each made on the host side so that no kernel
faults, traps or waits forever:

- RT_ERR_UNSUPPORTED: a scene feature outside the GPU path is refused by the
  world assembly (CPU, through rt_world_inspect; and on the GPU through
  rt_scene_create) rather than approximated;
- RT_ERR_STACK: a world whose traversal needs more stack entries than the
  kernels hold (the host computes the bound at build time) is refused before
  any launch, by every entry point that traces;
- RT_ERR_TIMEOUT: the wavefront's host-side iteration bound (the loop that
  polls the device) expires, forced with the test-only `iteration_limit`;
- RT_ERR_BOUNDS: the shadow queue fills up, forced with the test-only
  `shadow_queue_limit`; the kernel refuses the extra records and sets a flag
  the host reads.

After each refused or failed call the scene still renders correctly.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import rt

abi = rt.abi
S = rt.scenes

KERNEL_STACK_ENTRIES = 64   # the traversal stack every kernel holds (kStack)


def inspect_rc(pw):
    info = abi.RtSceneInfo()
    rc = abi.load().rt_world_inspect(pw.ref(), C.byref(info), None, 0, None, 0, None, 0)
    return rc, info


def unsupported_worlds():
    """(what, packed world) pairs the GPU path does not support."""
    out = []
    pw = abi.PackedWorld(S.cornell())
    pw.mats[0].type = 2                     # a material kind other than Disney / Emissive
    out.append(("material kind", pw))
    pw = abi.PackedWorld(S.cornell())
    pw.mats[1].thin_film_thickness = 400.0  # thin-film iridescence
    out.append(("thin film", pw))
    pw = abi.PackedWorld(S.cornell())
    pw.ents[2].kind = 7                     # an entity kind other than quad / sphere / mesh
    out.append(("entity kind", pw))
    w = S.throughput_scene(n_spheres=2, level=1)
    pw = abi.PackedWorld(w)
    pw.lights[0].type = 9                   # a light type other than area / directional / sphere
    out.append(("light type", pw))
    return out


@pytest.mark.parametrize("case", range(4))
def test_unsupported_features_are_refused_by_the_build(case):
    what, pw = unsupported_worlds()[case]
    rc, _ = inspect_rc(pw)
    assert rc == -6, what
    assert b"unsupported" in abi.load().rt_last_error() or b"outside" in abi.load().rt_last_error() or \
        b"only" in abi.load().rt_last_error()


def deep_world():
    """A mesh of 4000 tiny triangles at x = 1.02^i and 800 small spheres at
    y = 1.1^k: binned SAH peels a few items per level off both geometric
    sequences, so the top-level tree and the mesh tree are both deep, and the
    traversal needs more stack entries than the kernels hold."""
    w = S.World(name="deep")
    m = w.add_material("grey", S.disney((0.5, 0.5, 0.5)))
    rng = np.random.default_rng(5)
    n = 4000
    t = (rng.random((n, 9)) * 0.01).astype(np.float32)
    t[:, 0::3] += (1.02 ** np.arange(n, dtype=np.float64)).astype(np.float32)[:, None]
    w.add_mesh(t, m, name="expo")
    for k in range(800):
        w.add_sphere((0.0, float(1.1 ** k), 5.0), 0.01, m)
    w.camera = S.camera((0.0, 0.0, -30.0), (0.0, 0.0, 0.0))
    return w


def test_deep_world_needs_more_stack_than_the_kernels_hold():
    rc, info = inspect_rc(abi.PackedWorld(deep_world()))
    assert rc == 0 and info.top_is_bvh == 1
    assert info.max_stack_depth > KERNEL_STACK_ENTRIES


class _Scene:
    def __init__(self, world=None, packed=None):
        self.lib = abi.load()
        self.packed = packed or abi.PackedWorld(world)
        h = C.c_void_p()
        self.rc = self.lib.rt_scene_create(self.packed.ref(), C.byref(h))
        self.h = h

    def render(self, p):
        out = np.zeros((3, p.height, p.width), np.float32)
        st = abi.RtStats()
        rc = self.lib.rt_render(self.h, C.byref(p), abi.ptr(out), C.byref(st))
        return rc, out, st

    def close(self):
        if self.h:
            self.lib.rt_scene_destroy(self.h)


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(4))
def test_unsupported_features_are_refused_by_scene_create(case):
    what, pw = unsupported_worlds()[case]
    s = _Scene(packed=pw)
    assert s.rc == -6 and not s.h.value, what


@pytest.mark.gpu
def test_stack_bound_is_refused_before_launch():
    s = _Scene(deep_world())
    assert s.rc == 0
    try:
        for kernel in (abi.KERNEL_MEGAKERNEL, abi.KERNEL_WAVEFRONT):
            rc, _, _ = s.render(abi.render_params(16, 16, 1, 4, kernel=kernel))
            assert rc == -7 and b"stack" in s.lib.rt_last_error()
        rays = np.zeros((8, 8), np.float32)
        rays[:, 2] = -30.0
        rays[:, 5] = 1.0
        hits = np.zeros((8, 6), np.int32)
        assert s.lib.rt_trace_closest(s.h, abi.ptr(rays), 8, 1e-4, 3.4e38, abi.ptr(hits), 2) == -7
        tr = np.zeros((8, 3), np.float32)
        assert s.lib.rt_trace_any(s.h, abi.ptr(rays), 8, abi.ptr(tr), 2) == -7
        import torch
        film = torch.zeros((3, 16, 16), dtype=torch.float32, device="cuda")
        st = abi.RtStats()
        p = abi.render_params(16, 16, 1, 4, kernel=abi.KERNEL_MEGAKERNEL)
        assert s.lib.rt_render_device_noalloc(s.h, C.byref(p), C.c_void_p(film.data_ptr()), C.byref(st)) == -7
    finally:
        s.close()


@pytest.fixture(scope="module")
def cornell_scene():
    s = _Scene(S.cornell())
    assert s.rc == 0
    yield s
    s.close()


def _wf(**kw):
    return abi.render_params(48, 48, 64, 8, kernel=abi.KERNEL_WAVEFRONT, wavefront_size=1 << 12, **kw)


@pytest.mark.gpu
def test_iteration_bound_returns_timeout_and_the_scene_recovers(cornell_scene):
    s = cornell_scene
    ok_rc, ref, st = s.render(_wf())
    assert ok_rc == 0 and st.iterations > 8   # 147 456 samples through 4096 slots: many iterations
    rc, _, _ = s.render(_wf(iteration_limit=1))
    assert rc == -4 and b"iteration bound" in s.lib.rt_last_error()
    rc, again, _ = s.render(_wf())
    assert rc == 0
    np.testing.assert_allclose(again, ref, rtol=1e-4, atol=1e-6)


@pytest.mark.gpu
def test_full_shadow_queue_returns_bounds_and_the_scene_recovers(cornell_scene):
    s = cornell_scene
    ok_rc, ref, _ = s.render(_wf())
    assert ok_rc == 0
    rc, _, _ = s.render(_wf(shadow_queue_limit=64))
    assert rc == -5 and b"shadow queue" in s.lib.rt_last_error()
    rc, again, _ = s.render(_wf())
    assert rc == 0
    np.testing.assert_allclose(again, ref, rtol=1e-4, atol=1e-6)


@pytest.mark.gpu
def test_limits_that_are_not_reached_change_nothing(cornell_scene):
    """Generous limits leave the render as it is (the image is a function of
    the samples alone)."""
    s = cornell_scene
    _, ref, _ = s.render(_wf())
    rc, img, _ = s.render(_wf(iteration_limit=100000, shadow_queue_limit=1 << 20))
    assert rc == 0
    np.testing.assert_allclose(img, ref, rtol=1e-4, atol=1e-6)


@pytest.mark.gpu
def test_batch_limits_apply_to_the_whole_batch(cornell_scene):
    s = cornell_scene
    reqs = (abi.RtRequest * 2)()
    outs = [np.zeros((3, 32, 32), np.float32) for _ in range(2)]
    for i in range(2):
        reqs[i].scene, reqs[i].width, reqs[i].height, reqs[i].spp, reqs[i].max_depth = 0, 32, 32, 32, 8
        reqs[i].camera = abi.camera_desc(S.cornell().camera)
    scenes = (C.c_void_p * 1)(s.h)
    optrs = (C.c_void_p * 2)(*[o.ctypes.data for o in outs])
    st = abi.RtStats()
    common = abi.render_params(1, 1, 1, 1, kernel=abi.KERNEL_WAVEFRONT, wavefront_size=1 << 12, iteration_limit=2)
    assert s.lib.rt_render_batch(scenes, 1, reqs, 2, C.byref(common), optrs, C.byref(st)) == -4
    common.iteration_limit = 0
    abi.check(s.lib.rt_render_batch(scenes, 1, reqs, 2, C.byref(common), optrs, C.byref(st)), "rt_render_batch")
    assert all(np.all(np.isfinite(o)) and o.mean() > 0 for o in outs)
