"""The device SAH build (bvh_build.cu) against the host build and the oracle.

BvhNode's constructor (Acceleration/BvhNode.cs:91-364) fixes every node: the
16-bin SAH plane, the median fallbacks and the in-place partition's item
order. The device build must give the same nodes, boxes and leaf order bit
for bit (rt_scene_create_ex with RT_BVH_DEVICE, exported with
rt_scene_export_bvh), for the shapes that stress each part of it:

- long rotation chains in the partition (one right item ahead of many left ones);
- coincident centroids (median split, order kept) and flat axes (skipped);
- deep, unbalanced trees (many levels);
- meshes of 5..32 triangles (built whole by one thread);
- several meshes in one batch, lists of <= 4 triangles beside them.

CPU: the host build of the same meshes against the oracle, so that the
reference for the device comparison is itself pinned.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import rt

abi = rt.abi


def soup(n, seed, scale=10.0, size=0.3):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-scale, scale, (n, 1, 3))
    return (c + rng.normal(0, size, (n, 3, 3))).reshape(n, 9).astype(np.float32)


def chain(n):
    """Triangle 0 far along +x, the rest in [0, 1]: the root's partition has
    one right item ahead of n - 1 left ones, which rotates it n - 1 times."""
    t = soup(n, 7, scale=0.5, size=0.01)
    t[0, 0::3] += 1000.0
    return t


def coincident(n):
    """All centroids equal: no plane separates them (median split)."""
    rng = np.random.default_rng(3)
    d = rng.uniform(0.1, 1.0, (n, 1)).astype(np.float32)
    t = np.zeros((n, 9), np.float32)
    t[:, 0] = -d[:, 0]
    t[:, 3] = d[:, 0]
    t[:, 7] = 1.0
    t[:, 1] = -0.5
    t[:, 4] = -0.5
    t[:, 8] = 0.0
    t[:, 6] = 0.0
    return t


def flat(n):
    """Every triangle in the plane z = 0: the z axis has no extent."""
    t = soup(n, 11)
    t[:, 2::3] = 0.0
    return t


def exponential(n):
    """Centroids at 1.1^i along x: SAH peels a few items per level, so the
    tree is deep."""
    t = soup(n, 5, scale=0.0, size=0.01)
    t[:, 0::3] += (1.1 ** np.arange(n, dtype=np.float64)).astype(np.float32)[:, None]
    return t


def grid(n):
    """Centroids on an integer grid with repeats: many equal bin positions."""
    rng = np.random.default_rng(9)
    c = rng.integers(0, 6, (n, 1, 3)).astype(np.float32)
    return (c + np.array([[0, 0, 0], [0.5, 0, 0], [0, 0.5, 0.25]], np.float32)).reshape(n, 9)


def world_of(*meshes):
    w = rt.scenes.World()
    m = w.add_material("grey", rt.scenes.disney((0.5, 0.5, 0.5)))
    for k, t in enumerate(meshes):
        w.add_mesh(t, m, name=f"mesh{k}")
    w.camera = rt.scenes.camera((0.0, 0.0, -30.0), (0.0, 0.0, 0.0))
    return w


CASES = {
    "soup_1000": lambda: world_of(soup(1000, 1)),
    "soup_40000": lambda: world_of(soup(40000, 2)),
    "chain_5000": lambda: world_of(chain(5000)),
    "coincident_200": lambda: world_of(coincident(200)),
    "flat_3000": lambda: world_of(flat(3000)),
    "exponential_400": lambda: world_of(exponential(400)),
    "grid_5000": lambda: world_of(grid(5000)),
    "small_meshes": lambda: world_of(*[soup(n, 20 + n) for n in (5, 6, 7, 9, 16, 31, 32, 33, 34)]),
    "mixed_batch": lambda: world_of(soup(3, 40), soup(700, 41), chain(100), soup(4, 42), grid(2000), soup(12, 43),
                                    coincident(60), soup(20000, 44)),
}


def export(lib, h, info):
    nodes = np.zeros((info.num_nodes, 8), np.int32)
    top = np.zeros(max(info.num_entities, 1), np.int32)
    order = np.zeros(max(info.num_tris, 1), np.int32)
    abi.check(lib.rt_scene_export_bvh(h, abi.ptr(nodes), nodes.shape[0], abi.ptr(top), top.size, abi.ptr(order),
                                      order.size))
    return nodes, top, order


def host_inspect(world):
    lib = abi.load()
    pw = abi.PackedWorld(world)
    info = abi.RtSceneInfo()
    abi.check(lib.rt_world_inspect(pw.ref(), C.byref(info), None, 0, None, 0, None, 0), "rt_world_inspect")
    nodes = np.zeros((info.num_nodes, 8), np.int32)
    top = np.zeros(max(info.num_entities, 1), np.int32)
    order = np.zeros(max(info.num_tris, 1), np.int32)
    abi.check(lib.rt_world_inspect(pw.ref(), C.byref(info), abi.ptr(nodes), nodes.shape[0], abi.ptr(top), top.size,
                                   abi.ptr(order), order.size))
    return info, nodes, top, order


def device_scene(world, mode):
    lib = abi.load()
    pw = abi.PackedWorld(world)
    opt = abi.RtSceneOptions()
    opt.bvh_build = mode
    h = C.c_void_p()
    abi.check(lib.rt_scene_create_ex(pw.ref(), C.byref(opt), C.byref(h)), "rt_scene_create_ex")
    info = abi.RtSceneInfo()
    abi.check(lib.rt_scene_info(h, C.byref(info)))
    return lib, h, info, pw


# --- CPU: the host build of these meshes is the oracle's ----------------------------
@pytest.mark.parametrize("case", ["chain_5000", "coincident_200", "flat_3000", "exponential_400", "grid_5000",
                                  "small_meshes"])
def test_host_build_of_stress_meshes_matches_oracle(oracle, case):
    world = CASES[case]()
    info, nodes, _, order = host_inspect(world)
    osc = oracle.OracleScene(abi.PackedWorld(world))
    try:
        # mesh trees follow the top-level tree (or none when <= 4 entities)
        base = osc.export_top()[0].shape[0] if info.top_is_bvh else 0
        tri = 0
        for e, ent in enumerate(world.entities):
            onodes, oord = osc.export_mesh(e, ent["count"])
            assert np.array_equal(order[tri:tri + ent["count"]], oord[:ent["count"]])
            if ent["count"] > 4:
                got = nodes[base:base + onodes.shape[0]]
                box = np.concatenate([got[:, 0:3], got[:, 4:7]], 1)
                assert np.array_equal(box, onodes[:, 0:6])
                assert np.array_equal((got[:, 3] < 0).astype(np.int32), onodes[:, 6])
            base += max(onodes.shape[0], 1)
            tri += ent["count"]
    finally:
        osc.close()
    assert base == info.num_nodes


def _lomuto(items, left):
    """The host partition: each left item swaps with the first right one."""
    a, wp = list(items), 0
    for i in range(len(a)):
        if left[a[i]]:
            a[i], a[wp] = a[wp], a[i]
            wp += 1
    return a, wp


def _parallel(items, left):
    """The device formulation: left items at their rank; each right position
    follows p -> rank(p) while p holds a left item (pointer jumping)."""
    n = len(items)
    f = np.array([left[x] for x in items], bool)
    rank = np.concatenate([[0], np.cumsum(f)[:-1]]).astype(np.int64) if n else np.zeros(0, np.int64)
    nl = int(f.sum())
    ptr = np.where(f, rank, np.arange(n))
    for _ in range(max(1, int(np.ceil(np.log2(max(n, 2))))) + 1):
        ptr = ptr[ptr]
    out = [None] * n
    for p in range(n):
        if f[p]:
            out[rank[p]] = items[p]
        if p >= nl:
            out[p] = items[ptr[p]]
    return out, nl


def test_partition_rotation_formulation():
    rng = np.random.default_rng(0)
    for trial in range(3000):
        n = int(rng.integers(1, 60))
        left = rng.random(n) < rng.random()
        if trial % 5 == 0:                  # one right item ahead of n - 1 left ones
            left = np.ones(n, bool)
            left[0] = False
        items = list(range(n))
        assert _parallel(items, left) == _lomuto(items, left)


def test_scene_options_reject_bad_mode():
    lib = abi.load()
    opt = abi.RtSceneOptions()
    opt.bvh_build = 7
    h = C.c_void_p()
    rc = lib.rt_scene_create_ex(abi.PackedWorld(world_of(soup(10, 1))).ref(), C.byref(opt), C.byref(h))
    assert rc == -1   # RT_ERR_INVALID_ARG (checked before any device call)


# --- GPU: device build == host build, bit for bit -----------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(CASES))
def test_device_build_matches_host_build(case):
    world = CASES[case]()
    hinfo, hnodes, htop, horder = host_inspect(world)
    lib, h, info, _ = device_scene(world, abi.BVH_DEVICE)
    try:
        nodes, top, order = export(lib, h, info)
    finally:
        lib.rt_scene_destroy(h)
    assert info.bvh_on_device == 1
    assert info.num_nodes == hinfo.num_nodes
    np.testing.assert_array_equal(nodes, hnodes)
    np.testing.assert_array_equal(top, htop)
    np.testing.assert_array_equal(order, horder)
    assert info.max_stack_depth == hinfo.max_stack_depth


@pytest.mark.gpu
def test_device_build_of_the_bench_scene(throughput_world):
    """The 64 icospheres of the bench (1 310 722 triangles) built on the device
    equal the host build, and the device build is the automatic choice."""
    hinfo, hnodes, _, horder = host_inspect(throughput_world)
    lib, h, info, _ = device_scene(throughput_world, abi.BVH_AUTO)
    try:
        nodes, _, order = export(lib, h, info)
    finally:
        lib.rt_scene_destroy(h)
    assert info.bvh_on_device == 1
    np.testing.assert_array_equal(nodes, hnodes)
    np.testing.assert_array_equal(order, horder)


@pytest.mark.gpu
def test_auto_keeps_small_worlds_on_the_host(cornell_world):
    lib, h, info, _ = device_scene(cornell_world, abi.BVH_AUTO)
    lib.rt_scene_destroy(h)
    assert info.bvh_on_device == 0


@pytest.mark.gpu
def test_device_built_scene_renders_like_host_built():
    world = CASES["mixed_batch"]()
    world.add_sphere_light((0.0, 15.0, -5.0), 2.0, (1.0, 1.0, 1.0), 40.0)
    imgs = []
    for mode in ("host", "device"):
        r = rt.Renderer(world, 4, 4, kernel="wavefront", bvh_build=mode)
        try:
            assert r.info.bvh_on_device == (mode == "device")
            imgs.append(r.render(64, 48).beauty)
        finally:
            r.close()
    # the same tree traces the same paths; only the order of the film's float
    # atomics differs between runs
    np.testing.assert_allclose(imgs[0], imgs[1], rtol=1e-5, atol=1e-6)


@pytest.mark.gpu
def test_non_finite_vertex_falls_back_to_the_host():
    t = soup(100, 1)
    t[17, 4] = np.nan
    world = world_of(t)
    hinfo, hnodes, _, horder = host_inspect(world)
    lib, h, info, _ = device_scene(world, abi.BVH_DEVICE)
    try:
        nodes, _, order = export(lib, h, info)
    finally:
        lib.rt_scene_destroy(h)
    assert info.bvh_on_device == 0
    np.testing.assert_array_equal(nodes, hnodes)
    np.testing.assert_array_equal(order, horder)
