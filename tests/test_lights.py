"""Spherical emitters (§8(f) row 3): an emissive sphere as a GeometryLight
sampled in its solid-angle cone (Lights/GeometryLight.cs:202-238,
Geometry/Sphere.cs:108-226) and SphereLight (Lights/SphereLight.cs).

CPU: the host build derives the lights; in the oracle a SphereLight and an
emissive sphere of the same radiance light the box alike (both cone samplers
estimate the same radiance field); an observer inside an emissive sphere
takes the uniform-sphere fallback.
GPU: the scene with both emitters renders like the oracle.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import rt

abi = rt.abi


def rel_mse(x, r):
    return float(np.mean((x - r) ** 2 / (r ** 2 + 1e-2)))


def _info(world):
    info = abi.RtSceneInfo()
    rc = abi.load().rt_world_inspect(abi.PackedWorld(world).ref(), C.byref(info), None, 0, None, 0, None, 0)
    return rc, info


def test_host_build_derives_sphere_lights():
    rc, info = _info(rt.scenes.cornell_spheres())
    assert rc == 0
    # the ceiling quad and the emissive sphere (geometry lights) and the SphereLight
    assert info.num_lights == 3


def _sphere_emitter(kind: str):
    w = rt.scenes.cornell(tall_box=False)
    if kind == "light":
        w.add_sphere_light((278, 300, 278), 30.0, (1.0, 0.8, 0.6), 20.0, shadow_samples=4, name="bulb")
    else:   # an emissive sphere of the same radiance
        m = w.add_material("glow", rt.scenes.emissive((1.0, 0.8, 0.6), 20.0))
        w.add_sphere((278, 300, 278), 30.0, m, name="glow")
        w.geometry_light_samples = 4
    return w


def _oracle_render(oracle, world, w=32, h=32, spp=64, depth=8):
    osc = oracle.OracleScene(abi.PackedWorld(world))
    try:
        img, _ = osc.render(abi.render_params(w, h, spp, depth))
        return np.asarray(img, np.float64).reshape(3, h, w)
    finally:
        osc.close()


def test_oracle_sphere_light_equals_emissive_sphere(oracle):
    """The SphereLight's proxy emits colour x intensity and its NEE estimate is
    intensity x solid angle; an emissive sphere of that radiance is cone
    sampled with pdf 1 / solid angle. Both estimate one radiance field.
    The ceiling light is in both scenes, so compare the sphere's share: the
    difference to the scene without it."""
    base = _oracle_render(oracle, rt.scenes.cornell(tall_box=False))
    light = _oracle_render(oracle, _sphere_emitter("light")) - base
    geom = _oracle_render(oracle, _sphere_emitter("geometry")) - base
    assert light.mean() > 0.05 * base.mean()     # the sphere lights the box noticeably
    np.testing.assert_allclose(light.mean(axis=(1, 2)), geom.mean(axis=(1, 2)), rtol=0.05)


def _enclosed_world():
    """The box and camera inside a large emissive sphere, lit by a SphereLight
    inside it: every shading point is inside the emitter, so its cone sampler
    takes the uniform-sphere fallback (two more draws, pdf 1/4pi) and, the
    emitter facing outward, adds nothing; camera rays that leave the box see
    its back face, which does not emit."""
    w = rt.scenes.cornell(tall_box=False)
    m = w.add_material("shell", rt.scenes.emissive((0.5, 0.5, 0.5), 1.0))
    w.add_sphere((278, 278, 0), 2000.0, m, name="shell")
    w.add_sphere_light((278, 300, 278), 30.0, (1.0, 0.8, 0.6), 20.0, shadow_samples=4, name="bulb")
    w.geometry_light_samples = 2
    return w


def test_oracle_inside_an_emissive_sphere(oracle):
    img = _oracle_render(oracle, _enclosed_world(), 16, 16, 16)
    assert np.all(np.isfinite(img)) and img.max() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [abi.KERNEL_MEGAKERNEL, abi.KERNEL_WAVEFRONT])
def test_render_sphere_lights_match_oracle(oracle, kernel):
    from test_gpu_parity import Scene
    world = rt.scenes.cornell_spheres()
    s = Scene(world)
    try:
        g, st = s.render(abi.render_params(48, 48, 1024, 8, kernel=kernel, wavefront_size=1 << 16))
    finally:
        s.close()
    assert st.samples == 48 * 48 * 1024 and np.all(np.isfinite(g))
    o = _oracle_render(oracle, world, 48, 48, 256)
    np.testing.assert_allclose(g.mean(axis=(1, 2)), o.mean(axis=(1, 2)), rtol=0.02)
    assert rel_mse(o, g) < 0.05


@pytest.mark.gpu
def test_sphere_light_equals_emissive_sphere_on_gpu():
    from test_gpu_parity import Scene
    imgs = []
    for world in (rt.scenes.cornell(tall_box=False), _sphere_emitter("light"), _sphere_emitter("geometry")):
        s = Scene(world)
        try:
            imgs.append(s.render(abi.render_params(48, 48, 1024, 8, kernel=abi.KERNEL_WAVEFRONT))[0])
        finally:
            s.close()
    light, geom = imgs[1] - imgs[0], imgs[2] - imgs[0]
    np.testing.assert_allclose(light.mean(axis=(1, 2)), geom.mean(axis=(1, 2)), rtol=0.03)


@pytest.mark.gpu
def test_inside_an_emissive_sphere_matches_oracle(oracle):
    from test_gpu_parity import Scene
    world = _enclosed_world()
    s = Scene(world)
    try:
        g, _ = s.render(abi.render_params(32, 32, 1024, 8, kernel=abi.KERNEL_MEGAKERNEL))
    finally:
        s.close()
    o = _oracle_render(oracle, world, 32, 32, 256)
    np.testing.assert_allclose(g.mean(axis=(1, 2)), o.mean(axis=(1, 2)), rtol=0.03)


# --- the flat sky and its EnvironmentLight ----------------------------------------
def _sky_only(sky=(0.35, 0.45, 0.65)):
    """Nothing in view: one small quad behind the camera."""
    w = rt.scenes.World(name="sky-only")
    m = w.add_material("m", rt.scenes.disney((0.5, 0.5, 0.5)))
    w.add_quad((-1, -1, 10), (2, 0, 0), (0, 2, 0), m)
    w.sky = sky
    w.camera = rt.scenes.camera((0, 0, 0), (0, 0, -1), (0, 1, 0), 40.0)
    return w


def test_host_build_appends_the_environment_light():
    assert _info(rt.scenes.sky_scene())[1].num_lights == 1
    assert _info(rt.scenes.sky_scene(sky=(0.0, 0.0, 0.0)))[1].num_lights == 0
    assert _info(rt.scenes.sky_scene(sky=(1e-7, 0.0, 0.0)))[1].num_lights == 0   # luminance <= 1e-6: no NEE


def test_oracle_camera_rays_see_the_sky_at_full_weight(oracle):
    img = _oracle_render(oracle, _sky_only(), 8, 8, 4)
    np.testing.assert_allclose(img.mean(axis=(1, 2)), [0.35, 0.45, 0.65], rtol=1e-6)


def test_oracle_sky_mis_is_consistent(oracle):
    """The sky reaches a surface two ways, the EnvironmentLight's NEE and BSDF
    rays that miss; balance and power heuristics weight them differently but
    must estimate the same image."""
    w = rt.scenes.sky_scene()
    imgs = []
    for mis in (0, 1):   # RT_MIS_BALANCE, RT_MIS_POWER
        osc = oracle.OracleScene(abi.PackedWorld(w))
        try:
            img, _ = osc.render(abi.render_params(32, 24, 256, 6, mis_heuristic=mis))
            imgs.append(np.asarray(img, np.float64).reshape(3, 24, 32))
        finally:
            osc.close()
    np.testing.assert_allclose(imgs[0].mean(axis=(1, 2)), imgs[1].mean(axis=(1, 2)), rtol=0.02)


@pytest.mark.gpu
def test_camera_rays_see_the_sky_on_gpu():
    from test_gpu_parity import Scene
    s = Scene(_sky_only())
    try:
        for k in (abi.KERNEL_MEGAKERNEL, abi.KERNEL_WAVEFRONT):
            g, _ = s.render(abi.render_params(8, 8, 4, 8, kernel=k))
            np.testing.assert_allclose(g.mean(axis=(1, 2)), [0.35, 0.45, 0.65], rtol=1e-6)
    finally:
        s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [abi.KERNEL_MEGAKERNEL, abi.KERNEL_WAVEFRONT])
def test_render_sky_matches_oracle(oracle, kernel):
    """The sky term with its MIS weight, the EnvironmentLight's NEE (horizon
    test, unbounded shadow rays, glass transmittance) against the oracle."""
    from test_gpu_parity import Scene
    world = rt.scenes.sky_scene()
    s = Scene(world)
    try:
        g, st = s.render(abi.render_params(48, 32, 1024, 8, kernel=kernel, wavefront_size=1 << 16))
    finally:
        s.close()
    assert np.all(np.isfinite(g))
    o = _oracle_render(oracle, world, 48, 32, 256)
    np.testing.assert_allclose(g.mean(axis=(1, 2)), o.mean(axis=(1, 2)), rtol=0.02)
    assert rel_mse(o, g) < 0.05


# --- Power / Uniform light picking (LightDistribution, Renderer.cs:1907-1974) -------
def _two_suns():
    """Delta lights only: NEE carries no MIS weight, so picking one light per
    vertex (divided by its pick probability) estimates the same image as
    sampling every light."""
    w = rt.scenes.sky_scene(sky=(0.0, 0.0, 0.0))
    w.lights.append(dict(type=rt.scenes.LIGHT_DIRECTIONAL, direction=(-1.0, -2.0, -0.5), color=(1.0, 0.95, 0.9),
                         intensity=2.0, shadow_samples=1, angular_radius_deg=0.0))
    w.lights.append(dict(type=rt.scenes.LIGHT_DIRECTIONAL, direction=(1.5, -1.0, 0.5), color=(0.6, 0.7, 1.0),
                         intensity=0.7, shadow_samples=1, angular_radius_deg=0.0))
    return w


def _oracle_mean(oracle, world, strategy, w=32, h=24, spp=256):
    osc = oracle.OracleScene(abi.PackedWorld(world))
    try:
        img, _ = osc.render(abi.render_params(w, h, spp, 6, light_strategy=strategy))
        return np.asarray(img, np.float64).reshape(3, h, w)
    finally:
        osc.close()


def test_oracle_light_picking_is_unbiased_for_delta_lights(oracle):
    w = _two_suns()
    every = _oracle_mean(oracle, w, 0)
    for strategy in (1, 2):   # RT_LIGHTS_POWER, RT_LIGHTS_UNIFORM
        np.testing.assert_allclose(_oracle_mean(oracle, w, strategy).mean(axis=(1, 2)), every.mean(axis=(1, 2)),
                                   rtol=0.03)


@pytest.mark.gpu
@pytest.mark.parametrize("strategy,kernel", [(1, abi.KERNEL_MEGAKERNEL), (1, abi.KERNEL_WAVEFRONT),
                                             (2, abi.KERNEL_WAVEFRONT)])
def test_light_picking_matches_oracle(oracle, strategy, kernel):
    """Three non-delta emitters: the pick, its probability in the NEE MIS pdf
    and the division by it, as the oracle does them (including the reference's
    emission MIS, which keeps the unpicked light pdf)."""
    from test_gpu_parity import Scene
    world = rt.scenes.cornell_spheres()
    s = Scene(world)
    try:
        g, _ = s.render(abi.render_params(48, 48, 1024, 8, kernel=kernel, light_strategy=strategy,
                                          wavefront_size=1 << 16))
    finally:
        s.close()
    osc = oracle.OracleScene(abi.PackedWorld(world))
    try:
        o, _ = osc.render(abi.render_params(48, 48, 256, 8, light_strategy=strategy))
    finally:
        osc.close()
    o = np.asarray(o, np.float64).reshape(3, 48, 48)
    np.testing.assert_allclose(g.mean(axis=(1, 2)), o.mean(axis=(1, 2)), rtol=0.03)
    assert rel_mse(o, g) < 0.08


@pytest.mark.gpu
def test_unknown_light_strategy_is_rejected():
    from test_gpu_parity import Scene
    s = Scene(rt.scenes.cornell())
    try:
        out = np.zeros((3, 8, 8), np.float32)
        rc = s.lib.rt_render(s.h, C.byref(abi.render_params(8, 8, 1, 4, light_strategy=3)), abi.ptr(out),
                             C.byref(abi.RtStats()))
    finally:
        s.close()
    assert rc == -1   # RT_ERR_INVALID_ARG
