"""HDR film files and the capturing render (§8(f) row 2): PFM and EXR writers
(Rendering/PfmImage.cs, ExrImage.cs), RenderBuffers (RenderBuffers.cs) and
the AOV probe (Renderer.cs:755-882).

CPU: PFM/EXR layouts and round trips; the ZIP predictor; the oracle's capture
(A/B halves average to the beauty, B mirrors A at one sample, depth sentinel).
GPU: rt_render_capture against the oracle's capture, and its beauty against
rt_render's megakernel film.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np
import pytest

from conftest import rt

abi = rt.abi
images = rt.images


# --- PFM --------------------------------------------------------------------------
def test_pfm_layout_and_round_trip(tmp_path):
    rng = np.random.default_rng(1)
    rgb = rng.normal(size=(3, 5, 7)).astype(np.float32)
    p = str(tmp_path / "a.pfm")
    images.write_pfm(p, rgb, 7, 5, 3)
    data = open(p, "rb").read()
    head = b"PF\n7 5\n-1.0\n"
    assert data.startswith(head) and len(data) == len(head) + 4 * 3 * 35
    # the first stored row is the bottom one, channels interleaved
    first = np.frombuffer(data, "<f4", 3, len(head))
    np.testing.assert_array_equal(first, rgb[:, 4, 0])
    back, w, h, c = images.read_pfm(p)
    assert (w, h, c) == (7, 5, 3)
    np.testing.assert_array_equal(back, rgb)
    depth = rng.uniform(size=(5, 7)).astype(np.float32)
    images.write_pfm(p, depth, 7, 5, 1)
    assert open(p, "rb").read().startswith(b"Pf\n")
    np.testing.assert_array_equal(images.read_pfm(p)[0][0], depth)
    with pytest.raises(ValueError):
        images.write_pfm(p, depth, 7, 5, 2)


# --- EXR --------------------------------------------------------------------------
def test_zip_predictor_known_answer_and_inverse():
    raw = bytes([10, 20, 30, 40, 50])
    # split: even bytes then odd bytes, 10 30 50 20 40; then each byte minus the
    # one before it plus 128: 10, 148, 148, 20 - 50 + 128 = 98, 148
    assert images.zip_deconstruct(raw) == bytes([10, 148, 148, 98, 148])
    rng = np.random.default_rng(2)
    for n in (0, 1, 2, 7, 1000):
        b = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        assert images.zip_reconstruct(images.zip_deconstruct(b)) == b


def test_exr_header_and_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    w, h = 37, 41            # not a multiple of the 16-line block
    r = rng.normal(0, 100, (h, w)).astype(np.float32)
    r[0, 0], r[0, 1] = 1e6, -1e6          # clamp to the half range
    z = rng.uniform(size=(h, w)).astype(np.float32)
    p = str(tmp_path / "a.exr")
    images.write_exr(p, w, h, [("R", images.HALF, r), ("Z", images.FLOAT, z), ("B", images.HALF, r * 0.5)])
    data = open(p, "rb").read()
    assert struct.unpack_from("<Ii", data, 0) == (0x01312F76, 2)
    names = [b"channels", b"chromaticities", b"compression", b"dataWindow", b"displayWindow", b"lineOrder",
             b"pixelAspectRatio", b"screenWindowCenter", b"screenWindowWidth"]
    idx = [data.index(n + b"\0") for n in names]
    assert idx == sorted(idx)                               # the reference's attribute order
    ch = data.index(b"chlist\0") + 7 + 4
    assert data[ch:ch + 2] == b"B\0"                        # ordinal channel order: B, R, Z
    got = images.read_exr(p)
    np.testing.assert_array_equal(got["Z"], z)
    np.testing.assert_array_equal(got["R"], np.clip(r, -65504, 65504).astype(np.float16).astype(np.float32))
    np.testing.assert_array_equal(got["B"], (r * 0.5).clip(-65504, 65504).astype(np.float16).astype(np.float32))
    assert got["R"][0, 0] == 65504.0 and got["R"][0, 1] == -65504.0


def test_exr_stores_incompressible_blocks_raw(tmp_path):
    rng = np.random.default_rng(4)
    w, h = 64, 16
    noise = rng.integers(0, 2 ** 32, (h, w), dtype=np.uint32).view(np.float32)
    noise = np.where(np.isfinite(noise), noise, 0).astype(np.float32)
    p = str(tmp_path / "n.exr")
    images.write_exr(p, w, h, [("Y", images.FLOAT, noise)])
    data = open(p, "rb").read()
    (off,) = struct.unpack_from("<q", data, len(data) - (8 + w * h * 4) - 8)
    y, size = struct.unpack_from("<ii", data, off)
    assert (y, size) == (0, w * h * 4)                      # zlib did not shrink it: stored raw
    np.testing.assert_array_equal(images.read_exr(p)["Y"], noise)
    zlib.decompress(zlib.compress(b"x"))                    # zlib present


def test_exr_rejects_bad_channels(tmp_path):
    p = str(tmp_path / "x.exr")
    one = np.zeros((2, 2), np.float32)
    for chans in ([], [("R", 1, one), ("R", 1, one)], [("bad name", 1, one)], [("R", 1, np.zeros(3))]):
        with pytest.raises(ValueError):
            images.write_exr(p, 2, 2, chans)


# --- the capture in the oracle ------------------------------------------------------
def test_oracle_capture_halves_average_to_the_beauty(oracle, cornell_world):
    osc = oracle.OracleScene(abi.PackedWorld(cornell_world))
    try:
        p = abi.render_params(24, 24, 9, 8)
        cap = osc.render_capture(p)
        beauty, _ = osc.render(p)
    finally:
        osc.close()
    np.testing.assert_array_equal(cap["beauty"], beauty)       # the capture draws nothing extra
    buf = rt.RenderBuffers(24, 24, np.full(576, 9, np.int32), 5, 4, cap["beauty"], cap["beauty_a"],
                           cap["beauty_b"], cap["albedo_a"], cap["albedo_b"], cap["normal_a"], cap["normal_b"],
                           cap["depth_a"], cap["depth_b"])
    np.testing.assert_allclose(buf.combine_halves(buf.beauty_a, buf.beauty_b), beauty, rtol=1e-5, atol=1e-6)
    # the view is wider than the box at its opening: edge pixels whose samples
    # all missed keep the -1 sentinel, the others a positive mean distance
    d = cap["depth_a"]
    assert np.all((d > 0) | (d == -1)) and np.mean(d > 0) > 0.8
    comb = buf.combine_depth_halves()
    np.testing.assert_array_equal(comb < 0, (cap["depth_a"] < 0) & (cap["depth_b"] < 0))
    # diffuse walls: the albedo is the wall colour, the normal a unit vector
    n = np.linalg.norm(cap["normal_a"], axis=0)
    assert np.median(n) > 0.99 and cap["albedo_a"].max() <= 1.0
    assert np.all(buf.raw_beauty_variance() >= 0)


def test_oracle_capture_single_sample_mirrors_a_into_b(oracle, cornell_world):
    osc = oracle.OracleScene(abi.PackedWorld(cornell_world))
    try:
        cap = osc.render_capture(abi.render_params(8, 8, 1, 8))
    finally:
        osc.close()
    for k in ("beauty", "albedo", "normal", "depth"):
        np.testing.assert_array_equal(cap[f"{k}_a"], cap[f"{k}_b"])
    np.testing.assert_array_equal(cap["beauty_a"], cap["beauty"])


def test_renderbuffers_depth_sentinel():
    a = np.array([[-1, 2, -1, 4]], np.float32)
    b = np.array([[-1, -1, 3, 8]], np.float32)
    z = np.zeros((3, 1, 4), np.float32)
    buf = rt.RenderBuffers(4, 1, np.full(4, 4, np.int32), 2, 2, z, z, z, depth_a=a, depth_b=b)
    np.testing.assert_array_equal(buf.combine_depth_halves(), [[-1, 2, 3, 6]])


# --- GPU --------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("scene", ["cornell", "throughput", "volume"])
def test_gpu_capture_matches_oracle(oracle, scene):
    """Depth comes from the camera ray alone, so it agrees to rounding. Albedo
    and normal follow the delta-lobe chains, and beauty the whole path: those
    agree statistically (the same Sobol samples, different transcendental
    ulps)."""
    world = {"cornell": rt.scenes.cornell(), "throughput": rt.scenes.throughput_scene(n_spheres=8, level=3),
             "volume": rt.scenes.cornell_volume(density=0.3)}[scene]
    r = rt.Renderer(world, 64, 8, kernel="megakernel")
    try:
        res = r.render(48, 32, capture=rt.RenderCaptureOptions.FULL)
        plain = r.render(48, 32)
    finally:
        r.close()
    b = res.buffers
    assert b.has_aovs and b.samples_a == 32 and b.samples_b == 32
    osc = oracle.OracleScene(abi.PackedWorld(world))
    try:
        o = osc.render_capture(r.params(48, 32))
    finally:
        osc.close()
    # the capture traces the same paths as the plain megakernel
    np.testing.assert_allclose(res.beauty, plain.beauty, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(b.combine_halves(b.beauty_a, b.beauty_b), res.beauty, rtol=1e-5, atol=1e-6)
    for k in ("depth_a", "depth_b"):
        g, w = getattr(b, k), o[k]
        np.testing.assert_array_equal(g < 0, w < 0)
        np.testing.assert_allclose(g, w, rtol=1e-5)
    for k in ("albedo_a", "albedo_b", "normal_a", "normal_b"):
        g, w = getattr(b, k), o[k]
        np.testing.assert_allclose(g.mean(axis=(1, 2)), w.mean(axis=(1, 2)), atol=5e-3)
        assert np.mean(np.abs(g - w) < 1e-3) > 0.95, k       # per pixel: equal but for rare chain flips
    for k in ("beauty_a", "beauty_b"):
        np.testing.assert_allclose(getattr(b, k).mean(axis=(1, 2)), o[k].mean(axis=(1, 2)), rtol=0.03)


@pytest.mark.gpu
def test_capture_rejects_windows(cornell_world):
    import ctypes as C
    r = rt.Renderer(cornell_world, 4, 8, kernel="megakernel")
    try:
        p = r.params(32, 32, window_w=16, window_h=16)
        out = np.zeros((3, 32, 32), np.float32)
        rc = abi.load().rt_render_capture(r._scene, C.byref(p), abi.ptr(out), C.byref(abi.RtCapture()),
                                          C.byref(abi.RtStats()))
    finally:
        r.close()
    assert rc == -1   # RT_ERR_INVALID_ARG
