"""Smooth triangles (Geometry/SmoothTriangle.cs) and OBJ ingestion
(Scene/ObjLoader.cs, the direct path).

CPU: the OBJ loader's fan triangulation, index rules, dropped partial
channels, degenerate faces and float32 rounding; the host build's validation
of vertex normals; the oracle's smooth shading against its flat shading.
GPU: hits on smooth meshes and renders of a scene with a smooth anisotropic
sphere and a smooth emissive mesh against the oracle.
"""
from __future__ import annotations

import ctypes as C
import decimal

import numpy as np
import pytest

from conftest import random_rays, rt

abi = rt.abi
objfile = rt.objfile


def _write(tmp_path, text):
    p = tmp_path / "m.obj"
    p.write_text(text)
    return str(p)


def rel_mse(x, r):
    return float(np.mean((x - r) ** 2 / (r ** 2 + 1e-2)))


# --- OBJ ingestion --------------------------------------------------------------
def test_load_obj_fans_faces_and_resolves_indices(tmp_path):
    path = _write(tmp_path, """# a quad and a triangle
v 0 0 0
v 1 0 0
v 1 1 0
v 0 1 0
vt 0 0
vt 1 0
vt 1 1
vt 0 1
vn 0 0 1
vn 0 0 2
f 1/1/1 2/2/1 3/3/2 4/4/2
f -4/-4/-2 -2/-2/-1 -1/-1/-1
""")
    m = objfile.load_obj(path)
    assert m.warnings == []
    want = np.array([[0, 0, 0, 1, 0, 0, 1, 1, 0], [0, 0, 0, 1, 1, 0, 0, 1, 0], [0, 0, 0, 1, 1, 0, 0, 1, 0]],
                    np.float32)
    np.testing.assert_array_equal(m.tris, want)
    np.testing.assert_array_equal(m.normals[0], [0, 0, 1, 0, 0, 1, 0, 0, 2])
    np.testing.assert_array_equal(m.normals[2], [0, 0, 1, 0, 0, 2, 0, 0, 2])
    np.testing.assert_array_equal(m.uvs[1], [0, 0, 1, 1, 0, 1])


def test_load_obj_drops_partial_channels_and_skips_degenerate_faces(tmp_path):
    path = _write(tmp_path, """v 0 0 0
v 1 0 0
v 0 1 0
v 2 0 0
vn 0 0 1
f 1//1 2//1 3//1
f 1 2 3
f 1 2 4
f 1 2
v 1\t2 3
f 1 9 2
""")
    m = objfile.load_obj(path)
    # the second face has no normals: the whole mesh is flat (ObjLoader.cs:205-208)
    assert m.normals is None and m.uvs is None
    # the collinear face is skipped, and so is the face with two vertices
    assert m.tris.shape == (2, 9)
    assert any("fewer than 3" in w for w in m.warnings)
    assert any("malformed vertex position" in w for w in m.warnings)
    assert any("malformed face vertex '9'" in w for w in m.warnings)


def test_float_parse_rounds_once_to_float32():
    """A decimal just above the midpoint of two float32 neighbours reads as a
    float64 exactly on the midpoint; ties-to-even would then give the lower
    neighbour, but the correctly rounded float32 is the upper one."""
    decimal.getcontext().prec = 100
    exact = decimal.Decimal(1) + decimal.Decimal(2) ** -24 + decimal.Decimal(2) ** -60
    s = str(exact)
    assert np.float32(float(s)) == np.float32(1.0)          # the double-rounding trap
    assert objfile._f32([s])[0] == np.nextafter(np.float32(1), np.float32(2))
    below = str(decimal.Decimal(1) + decimal.Decimal(2) ** -24 - decimal.Decimal(2) ** -60)
    assert objfile._f32([below])[0] == np.float32(1.0)
    assert objfile._f32(["0.1", "-2.5e-3", "1e38"]).tolist() == np.array([0.1, -2.5e-3, 1e38], np.float32).tolist()


def test_obj_round_trip_is_exact(tmp_path):
    tris, nn, uv = rt.scenes.smooth_icosphere(2, (1.5, -2.0, 3.25), 0.7)
    p = str(tmp_path / "s.obj")
    objfile.write_obj(p, tris, nn, uv)
    m = objfile.load_obj(p)
    np.testing.assert_array_equal(m.tris, tris)
    np.testing.assert_array_equal(m.normals, nn)
    np.testing.assert_array_equal(m.uvs, uv)
    w = rt.scenes.World()
    w.add_obj(p, w.add_material("m", rt.scenes.disney((0.5, 0.5, 0.5))))
    np.testing.assert_array_equal(w.tri_normals, nn)


def test_yaml_export_writes_smooth_meshes(tmp_path):
    w = rt.scenes.cornell_smooth()
    rt.scenes.write_yaml(w, str(tmp_path))
    i = [e["name"] for e in w.entities].index("smooth_sphere")
    m = objfile.load_obj(str(tmp_path / f"{w.name}_{i}.obj"))
    e = w.entities[i]
    np.testing.assert_array_equal(m.normals, w.tri_normals[e["first"]:e["first"] + e["count"]])


# --- host build -----------------------------------------------------------------
def _inspect(world):
    lib = abi.load()
    info = abi.RtSceneInfo()
    return lib.rt_world_inspect(abi.PackedWorld(world).ref(), C.byref(info), None, 0, None, 0, None, 0)


def test_host_build_accepts_smooth_and_rejects_bad_normals():
    w = rt.scenes.cornell_smooth()
    assert _inspect(w) == 0
    bad = rt.scenes.cornell_smooth()
    bad.tri_normals = bad.tri_normals.copy()
    e = [x for x in bad.entities if x["name"] == "smooth_sphere"][0]
    bad.tri_normals[e["first"] + 5, 3:6] = 0.0          # one zero vertex normal
    assert _inspect(bad) == -1   # RT_ERR_INVALID_ARG
    bad.tri_normals[e["first"] + 5, 3:6] = np.nan
    assert _inspect(bad) == -1   # RT_ERR_INVALID_ARG


# --- oracle ---------------------------------------------------------------------
def _oracle_render(oracle, world, w=32, h=32, spp=64):
    osc = oracle.OracleScene(abi.PackedWorld(world))
    try:
        img, _ = osc.render(abi.render_params(w, h, spp, 8))
        return np.asarray(img, np.float64).reshape(3, h, w)
    finally:
        osc.close()


def _sphere_world(normals: str):
    w = rt.scenes.cornell(tall_box=False)
    m = w.add_material("aniso", rt.scenes.disney((0.8, 0.6, 0.3), roughness=0.3, metallic=0.7, anisotropic=0.8))
    tris, nn, _ = rt.scenes.smooth_icosphere(2, (370, 100, 350), 100.0, with_uvs=False)
    if normals == "flat":
        w.add_mesh(tris, m)
    else:
        if normals == "face":   # every vertex carries the face normal
            t = tris.reshape(-1, 3, 3).astype(np.float64)
            fn = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
            fn /= np.linalg.norm(fn, axis=1, keepdims=True)
            nn = np.repeat(fn, 3, axis=0).reshape(-1, 9).astype(np.float32)
        w.add_mesh(tris, m, normals=nn)
    return w


def test_oracle_smooth_with_face_normals_shades_like_flat(oracle):
    """Vertex normals equal to the face normal interpolate back to it (to
    rounding), and the default UVs give the flat triangle's edge frame: the
    image is the flat mesh's."""
    flat = _oracle_render(oracle, _sphere_world("flat"))
    face = _oracle_render(oracle, _sphere_world("face"))
    np.testing.assert_allclose(face.mean(axis=(1, 2)), flat.mean(axis=(1, 2)), rtol=1e-3)
    assert rel_mse(face, flat) < 1e-3


def test_oracle_smooth_normals_change_the_shading(oracle):
    flat = _oracle_render(oracle, _sphere_world("flat"))
    smooth = _oracle_render(oracle, _sphere_world("smooth"))
    assert rel_mse(smooth, flat) > 5e-4   # 2.4e-3 measured; face normals give 6e-7


# --- GPU ------------------------------------------------------------------------
@pytest.mark.gpu
def test_smooth_mesh_hits_match_oracle(oracle):
    """Smooth triangles intersect exactly like flat ones (SmoothTriangle.Hit
    reuses Moller-Trumbore): primitive ids and t equal the oracle's."""
    from test_gpu_parity import Scene, _compare_hits
    world = rt.scenes.cornell_smooth()
    s = Scene(world)
    try:
        rays = random_rays(((1, 1, 1), (554, 554, 554)), 50000, seed=31)
        _compare_hits(s.closest(rays), oracle.OracleScene(abi.PackedWorld(world)).trace_closest(rays)[0])
    finally:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [abi.KERNEL_MEGAKERNEL, abi.KERNEL_WAVEFRONT])
def test_render_smooth_matches_oracle(oracle, kernel):
    """Interpolated shading normals, the UV tangent frame of an anisotropic
    lobe, and a smooth emissive mesh's light samples and pdf: the GPU image
    estimates the oracle's."""
    from test_gpu_parity import Scene
    world = rt.scenes.cornell_smooth()
    s = Scene(world)
    try:
        g, st = s.render(abi.render_params(48, 48, 1024, 8, kernel=kernel, wavefront_size=1 << 16))
    finally:
        s.close()
    assert st.samples == 48 * 48 * 1024 and np.all(np.isfinite(g))
    o = _oracle_render(oracle, world, 48, 48, 256)
    np.testing.assert_allclose(g.mean(axis=(1, 2)), o.mean(axis=(1, 2)), rtol=0.02)
    assert rel_mse(o, g) < 0.05
    flat = rt.scenes.cornell_smooth()
    flat.tri_normals = np.zeros_like(flat.tri_normals)   # every triangle flat
    f = _oracle_render(oracle, flat, 48, 48, 256)
    assert rel_mse(f, g) > 2 * rel_mse(o, g)   # the smooth shading is what matches
