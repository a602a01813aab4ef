"""Host-side world assembly (librt3d.so, no GPU needed) against the oracle:
the binned-SAH BVH (Acceleration/BvhNode.cs:91-364) must come out node for
node identical, boxes bit-exact, and the RR classifier must agree."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import rt

abi = rt.abi


def inspect(world):
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


def decode(nodes):
    """-> (box words [n,6], leaf flag, axis or -1, first, count)"""
    box = np.concatenate([nodes[:, 0:3], nodes[:, 4:7]], 1)
    a, b = nodes[:, 3], nodes[:, 7]
    leaf = (a < 0).astype(np.int32)
    axis = np.where(leaf == 0, (b.view(np.uint32) >> 30).astype(np.int32), 0)
    first = np.where(leaf == 1, ~a, 0)
    count = np.where(leaf == 1, b & 0xFFFF, 0)
    return box, leaf, axis, first, count


def compare_tree(prod_nodes, base, or_nodes, item_base=0, is_list=False):
    n = or_nodes.shape[0]
    box, leaf, axis, first, count = decode(prod_nodes[base:base + max(n, 1)])
    if is_list:
        return
    assert np.array_equal(box, or_nodes[:, 0:6]), "node boxes differ"
    assert np.array_equal(leaf, or_nodes[:, 6])
    assert np.array_equal(axis[leaf == 0], or_nodes[or_nodes[:, 6] == 0, 7])
    assert np.array_equal(first[leaf == 1] - item_base, or_nodes[or_nodes[:, 6] == 1, 8])
    assert np.array_equal(count[leaf == 1], or_nodes[or_nodes[:, 6] == 1, 9])


@pytest.mark.parametrize("which", ["cornell", "throughput_small", "sphere", "volume"])
def test_bvh_matches_oracle(oracle, which, cornell_world, throughput_world_small):
    world = {"cornell": cornell_world, "throughput_small": throughput_world_small,
             "sphere": rt.scenes.cornell_sphere(), "volume": rt.scenes.cornell_volume()}[which]
    info, nodes, top, order = inspect(world)
    osc = oracle.OracleScene(abi.PackedWorld(world))
    oi = osc.info()
    assert info.top_is_bvh == oi["top_is_bvh"]
    assert info.num_lights == oi["num_lights"]
    assert info.rr_min_bounces == oi["rr_min_bounces"]
    assert np.float32(info.rr_min_survival) == np.float32(oi["rr_min_survival"])
    assert np.float32(info.mean_irradiance) == np.float32(oi["mean_irradiance"])
    base = 0
    if info.top_is_bvh:
        otop, oorder = osc.export_top()
        compare_tree(nodes, 0, otop)
        assert np.array_equal(top[:len(world.entities)], oorder[:len(world.entities)])
        base = otop.shape[0]
    tri_base = 0
    for e, ent in enumerate(world.entities):
        if ent["kind"] != rt.scenes.ENT_MESH:
            continue
        onodes, oord = osc.export_mesh(e, ent["count"])
        is_list = ent["count"] <= 4
        compare_tree(nodes, base, onodes, tri_base, is_list)
        assert np.array_equal(order[tri_base:tri_base + ent["count"]], oord[:ent["count"]])
        base += max(onodes.shape[0], 1)
        tri_base += ent["count"]
    assert base == info.num_nodes
    assert tri_base == info.num_tris


def test_full_throughput_scene_sizes(throughput_world):
    """C2 at full size: 64 level-5 icospheres + a 2-triangle ground."""
    assert throughput_world.num_tris == 64 * 20480 + 2
    info, _, _, _ = inspect(throughput_world)
    assert info.num_tris == throughput_world.num_tris
    assert info.max_stack_depth <= 64
    assert info.rr_min_bounces == 3   # direct-dominant (sun + area light)


def test_cornell_classifier_is_indirect_dominant(cornell_world):
    """Renderer.cs:361-378: mean irradiance ~0.18 < 0.5 -> RR from bounce 6, min survival 0.4."""
    info, _, _, _ = inspect(cornell_world)
    assert info.rr_min_bounces == 6
    assert abs(info.rr_min_survival - 0.4) < 1e-7
    assert 0.17 < info.mean_irradiance < 0.19


def test_energy_lut_bit_exact(oracle, lib):
    e = np.zeros(1024, np.float32)
    ea = np.zeros(32, np.float32)
    abi.check(lib.rt_energy_lut(abi.ptr(e), abi.ptr(ea)))
    oe, oea = oracle.energy_lut()
    assert np.array_equal(e.view(np.uint32), oe.view(np.uint32))
    assert np.array_equal(ea.view(np.uint32), oea.view(np.uint32))
    assert np.all((e >= 0) & (e <= 1)) and np.all(np.diff(ea) <= 1e-6)   # E_avg falls with roughness


def test_invalid_world_is_rejected(lib):
    w = rt.scenes.cornell()
    w.entities[0]["material"] = 99
    info = abi.RtSceneInfo()
    rc = lib.rt_world_inspect(abi.PackedWorld(w).ref(), C.byref(info), None, 0, None, 0, None, 0)
    assert rc == -1 and b"material" in lib.rt_last_error()
