"""Host-side mirror of 3d-ray's `Renderer` API over the C-ABI.

`Renderer(world, ...)` takes the constructor arguments of
src/RayTracer/Rendering/Renderer.cs:300-319 that matter on the GPU path and
`render(width, height)` returns a `RenderResult` like Renderer.Render
(:522-733): display pixels (ACES + gamma, [H, W, 3]) and the linear-HDR
beauty buffer (planar [3, H, W], the FrameBuffer layout). Everything below
the call runs in librt3d.so on the GPU; there is no CPU fallback — a missing
library or device raises.

The reference's `world` is an IHittable graph built by its YAML loader; here
it is a `scenes.World` (the same information, entity-level), from which the
library performs the world assembly and SAH build.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import abi, scenes

MIS = {"balance": 0, "power": 1}
BVH_BUILD = {"auto": 0, "host": 1, "device": 2}   # RT_BVH_*: where the mesh BVHs are built
LIGHT_STRATEGY = {"all": 0, "power": 1, "uniform": 2}   # RT_LIGHTS_*
KERNELS = {"megakernel": abi.KERNEL_MEGAKERNEL, "wavefront": abi.KERNEL_WAVEFRONT}


@dataclasses.dataclass(frozen=True)
class RenderCaptureOptions:
    """Which side buffers a render captures (Rendering/RenderBuffers.cs:9-23)."""
    capture_beauty_halves: bool = False
    capture_aovs: bool = False

    @property
    def any(self) -> bool:
        return self.capture_beauty_halves or self.capture_aovs


RenderCaptureOptions.NONE = RenderCaptureOptions()
RenderCaptureOptions.FULL = RenderCaptureOptions(True, True)


@dataclasses.dataclass
class RenderBuffers:
    """Linear-HDR frame data of a capturing render (RenderBuffers.cs:50-169):
    every quantity split by sample-index parity into A (the ceil(n/2) even
    samples) and B (the floor(n/2) odd ones), each a mean; B mirrors A when
    n == 1. Depth is the world-space distance to the camera ray's first hit,
    -1 where no sample of the half hit geometry. Colour planes are [3, H, W],
    depth [H, W]."""
    width: int
    height: int
    sample_count: np.ndarray     # [H * W] int32 (uniform)
    samples_a: int
    samples_b: int
    beauty: np.ndarray
    beauty_a: np.ndarray
    beauty_b: np.ndarray
    albedo_a: np.ndarray | None = None
    albedo_b: np.ndarray | None = None
    normal_a: np.ndarray | None = None
    normal_b: np.ndarray | None = None
    depth_a: np.ndarray | None = None
    depth_b: np.ndarray | None = None

    @property
    def has_aovs(self) -> bool:
        return self.albedo_a is not None

    def combine_halves(self, a: np.ndarray, b: np.ndarray) -> np.ndarray:
        """(nA * A + nB * B) / n (:101-118)."""
        n = self.samples_a + self.samples_b
        if self.samples_b == 0:
            return a.copy()
        wa = np.float32(np.float32(self.samples_a) / np.float32(n))
        wb = np.float32(np.float32(self.samples_b) / np.float32(n))
        return (wa * a.astype(np.float32) + wb * b.astype(np.float32)).astype(np.float32)

    def combine_depth_halves(self) -> np.ndarray:
        """Sentinel-aware depth combination (:125-150)."""
        if self.depth_a is None:
            raise ValueError("Depth AOV was not captured.")
        n = self.samples_a + self.samples_b
        wa = np.float32(np.float32(self.samples_a) / np.float32(n)) if n > 0 else np.float32(1.0)
        wb = np.float32(np.float32(1.0) - wa)
        a, b = self.depth_a.astype(np.float32), self.depth_b.astype(np.float32)
        both = a * wa + b * wb if self.samples_b else a
        out = np.where(a < 0, np.where(b < 0, np.float32(-1.0), b), np.where(b < 0, a, both))
        return out.astype(np.float32)

    def raw_beauty_variance(self) -> np.ndarray:
        """((A - B) / 2)^2 per channel (:157-168)."""
        d = np.float32(0.5) * (self.beauty_a.astype(np.float32) - self.beauty_b.astype(np.float32))
        return (d * d).astype(np.float32)


@dataclasses.dataclass
class RenderResult:
    pixels: np.ndarray        # [H, W, 3] display RGB in [0, 1]
    beauty: np.ndarray        # [3, H, W] linear HDR (mean of clamped samples)
    stats: dict
    buffers: RenderBuffers | None = None


class Renderer:
    DEFAULT_MAX_SAMPLE_RADIANCE = 10.0    # Renderer.cs:202
    DEFAULT_INDIRECT_CLAMP_FACTOR = 0.25  # Renderer.cs:214

    def __init__(self, world: "scenes.World", samples_per_pixel: int, max_depth: int,
                 max_sample_radiance: float | None = None, verbose: bool = False,
                 mis_heuristic: str = "balance", light_sampling_strategy: str = "all",
                 indirect_clamp_factor: float = DEFAULT_INDIRECT_CLAMP_FACTOR, exposure_ev: float = 0.0,
                 kernel: str = "wavefront", bvh_build: str = "auto"):
        if light_sampling_strategy not in LIGHT_STRATEGY:
            raise ValueError(f"unknown light strategy {light_sampling_strategy!r}")
        self.world = world
        self.spp = int(samples_per_pixel)
        self.max_depth = int(max_depth)
        self.max_sample_radiance = self.DEFAULT_MAX_SAMPLE_RADIANCE if max_sample_radiance is None \
            else float(max_sample_radiance)
        self.indirect_clamp_factor = float(indirect_clamp_factor)
        self.exposure_ev = float(exposure_ev)
        self.mis = MIS[mis_heuristic]
        self.light_strategy = LIGHT_STRATEGY[light_sampling_strategy]
        self.kernel = KERNELS[kernel]
        self.verbose = verbose
        self._lib = abi.load()
        self._packed = abi.PackedWorld(world)
        h = C.c_void_p()
        opt = abi.RtSceneOptions()
        opt.bvh_build = BVH_BUILD[bvh_build]
        abi.check(self._lib.rt_scene_create_ex(self._packed.ref(), C.byref(opt), C.byref(h)), "rt_scene_create_ex")
        self._scene = h
        info = abi.RtSceneInfo()
        abi.check(self._lib.rt_scene_info(h, C.byref(info)))
        self.info = info
        if verbose and info.rr_min_bounces == 6:
            print("  Lighting:    indirect-dominant (conservative RR)")

    def close(self):
        if getattr(self, "_scene", None):
            self._lib.rt_scene_destroy(self._scene)
            self._scene = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self, width: int, height: int, **kw) -> "abi.RtRenderParams":
        return abi.render_params(width, height, self.spp, self.max_depth,
                                 max_sample_radiance=self.max_sample_radiance,
                                 indirect_clamp_factor=self.indirect_clamp_factor, exposure_ev=self.exposure_ev,
                                 mis_heuristic=self.mis, light_strategy=self.light_strategy, kernel=self.kernel,
                                 **kw)

    def autotune(self, width: int, height: int) -> dict:
        best = abi.RtRenderParams()
        p = self.params(width, height)
        abi.check(self._lib.rt_autotune(self._scene, C.byref(p), C.byref(best)), "rt_autotune")
        return dict(wavefront_size=best.wavefront_size, block_size=best.block_size,
                    sort_materials=best.sort_materials)

    def render(self, width: int, height: int, capture: RenderCaptureOptions | None = None, **kw) -> RenderResult:
        """Renderer.Render(w, h[, RenderCaptureOptions]). A capture runs the
        plain megakernel (rt_render_capture) and fills `buffers`."""
        p = self.params(width, height, **kw)
        beauty = np.zeros((3, height, width), np.float32)
        st = abi.RtStats()
        bufs = None
        if capture is not None and capture.any:
            planes = {k: np.zeros((3, height, width), np.float32) for k in ("beauty_a", "beauty_b")}
            if capture.capture_aovs:
                for k in ("albedo_a", "albedo_b", "normal_a", "normal_b"):
                    planes[k] = np.zeros((3, height, width), np.float32)
                for k in ("depth_a", "depth_b"):
                    planes[k] = np.zeros((height, width), np.float32)
            cap = abi.RtCapture(**{k: v.ctypes.data for k, v in planes.items()})
            abi.check(self._lib.rt_render_capture(self._scene, C.byref(p), abi.ptr(beauty), C.byref(cap),
                                                  C.byref(st)), "rt_render_capture")
            bufs = RenderBuffers(width, height, np.full(width * height, self.spp, np.int32), (self.spp + 1) // 2,
                                 self.spp // 2, beauty, **planes)
        else:
            abi.check(self._lib.rt_render(self._scene, C.byref(p), abi.ptr(beauty), C.byref(st)), "rt_render")
        return RenderResult(self.tone_map_to_display(beauty), beauty,
                            {f: getattr(st, f) for f, _ in abi.RtStats._fields_}, bufs)

    def tone_map_to_display(self, beauty: np.ndarray) -> np.ndarray:
        """Renderer.ToneMapToDisplay (:741): exposure, ACES, gamma on the GPU."""
        _, h, w = beauty.shape
        beauty = np.ascontiguousarray(beauty, np.float32)
        out = np.zeros((h, w, 3), np.float32)
        abi.check(self._lib.rt_tonemap(abi.ptr(beauty), w, h, self.exposure_ev, abi.ptr(out)), "rt_tonemap")
        return out


def render_batch(requests, worlds, common_kernel: str = "wavefront", **kw):
    """Renders many (scene, camera, size, spp, depth) requests in one
    persistent wavefront launch (rt_render_batch). `worlds` is a list of
    scenes.World; each request is a dict with scene (index), width, height,
    spp, max_depth and camera (scenes.camera dict). Returns the linear-HDR
    films and the stats."""
    lib = abi.load()
    packed = [abi.PackedWorld(w) for w in worlds]
    handles = []
    try:
        for pw in packed:
            h = C.c_void_p()
            abi.check(lib.rt_scene_create(pw.ref(), C.byref(h)), "rt_scene_create")
            handles.append(h)
        n = len(requests)
        reqs = (abi.RtRequest * n)()
        outs = []
        for i, r in enumerate(requests):
            q = reqs[i]
            q.scene, q.width, q.height, q.spp, q.max_depth = r["scene"], r["width"], r["height"], r["spp"], \
                r["max_depth"]
            q.camera = abi.camera_desc(r["camera"])
            outs.append(np.zeros((3, r["height"], r["width"]), np.float32))
        common = abi.render_params(1, 1, 1, 1, kernel=KERNELS[common_kernel], **kw)
        st = abi.RtStats()
        arr = (C.c_void_p * len(handles))(*[h.value for h in handles])
        optrs = (C.c_void_p * n)(*[o.ctypes.data for o in outs])
        abi.check(lib.rt_render_batch(arr, len(handles), reqs, n, C.byref(common), optrs, C.byref(st)),
                  "rt_render_batch")
        return outs, st
    finally:
        for h in handles:
            lib.rt_scene_destroy(h)
