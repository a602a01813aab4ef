"""Every constructor argument the `Renderer` mirror forwards to the GPU
(Rendering/Renderer.cs:300-333: maxSampleRadiance, misHeuristic,
lightSamplingStrategy, indirectClampFactor, exposureEv) reaches the kernels
and changes the image the way it changes the oracle's.

For each knob the scene is rendered through `rt.Renderer` on both kernels and
by the oracle with the same settings: the GPU image must differ from the
default-settings image (the knob was not dropped on the way), and must match
the oracle's image for that setting (channel means within 2%, relMSE < 0.05).
The exposure only enters the display transform: the HDR film is unchanged and
the display pixels equal the oracle's tone map of it at that exposure.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rt

abi = rt.abi
W = H = 32
SPP_GPU = 1024
SPP_ORACLE = 256

KNOBS = {
    "default": {},
    "max_sample_radiance": dict(max_sample_radiance=1.5),
    "indirect_clamp_factor": dict(indirect_clamp_factor=0.02),
    "mis_power": dict(mis_heuristic="power"),
    "lights_power": dict(light_sampling_strategy="power"),
    "lights_uniform": dict(light_sampling_strategy="uniform"),
}


def rel_mse(x, r):
    return float(np.mean((x - r) ** 2 / (r ** 2 + 1e-2)))


def oracle_image(oracle, world, kw):
    p = abi.render_params(W, H, SPP_ORACLE, 8,
                          max_sample_radiance=kw.get("max_sample_radiance", 10.0),
                          indirect_clamp_factor=kw.get("indirect_clamp_factor", 0.25),
                          mis_heuristic=rt.renderer.MIS[kw.get("mis_heuristic", "balance")],
                          light_strategy=rt.renderer.LIGHT_STRATEGY[kw.get("light_sampling_strategy", "all")])
    img, _ = oracle.OracleScene(abi.PackedWorld(world)).render(p)
    return img


@pytest.fixture(scope="module")
def world():
    return rt.scenes.cornell_spheres()


@pytest.fixture(scope="module")
def default_images(world):
    out = {}
    for kernel in ("megakernel", "wavefront"):
        r = rt.Renderer(world, SPP_GPU, 8, kernel=kernel)
        try:
            out[kernel] = r.render(W, H).beauty
        finally:
            r.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["megakernel", "wavefront"])
@pytest.mark.parametrize("knob", [k for k in KNOBS if k != "default"])
def test_forwarded_knob_changes_the_image_as_in_the_oracle(oracle, world, default_images, knob, kernel):
    kw = KNOBS[knob]
    r = rt.Renderer(world, SPP_GPU, 8, kernel=kernel, **kw)
    try:
        g = r.render(W, H).beauty
    finally:
        r.close()
    assert not np.array_equal(g, default_images[kernel]), f"{knob} did not reach the kernel"
    o = oracle_image(oracle, world, kw)
    np.testing.assert_allclose(g.mean(axis=(1, 2)), o.mean(axis=(1, 2)), rtol=0.02)
    assert rel_mse(o, g) < 0.05


@pytest.mark.gpu
def test_exposure_changes_the_display_pixels_only(oracle, world, default_images):
    r = rt.Renderer(world, SPP_GPU, 8, kernel="wavefront", exposure_ev=1.5)
    try:
        res = r.render(W, H)
    finally:
        r.close()
    np.testing.assert_allclose(res.beauty, default_images["wavefront"], rtol=1e-4, atol=1e-6)
    np.testing.assert_allclose(res.pixels, oracle.tonemap(res.beauty, 1.5), rtol=2e-6, atol=1e-7)
    assert np.mean(res.pixels) > np.mean(oracle.tonemap(res.beauty, 0.0))
