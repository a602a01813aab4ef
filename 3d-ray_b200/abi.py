"""ctypes mirror of include/rt3d.h and the loader for the in-tree librt3d.so.

The shared library is the product: CUDA kernels for sm_100a plus the host-side
world assembly, behind a plain C ABI (the same entry points a .NET P/Invoke
shim binds). `load()` fails loudly when the library is missing — there is no
CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import scenes

HERE = os.path.dirname(os.path.abspath(__file__))
# RT3D_LIB selects another build of the same ABI, e.g. lib/librt3d_checked.so
# (every kernel index range-checked) for a run of the test suite.
LIB_PATH = os.environ.get("RT3D_LIB") or os.path.join(HERE, "lib", "librt3d.so")
CHECKED_LIB_PATH = os.path.join(HERE, "lib", "librt3d_checked.so")

RT_OK = 0
ERRORS = {-1: "RT_ERR_INVALID_ARG", -2: "RT_ERR_OOM", -3: "RT_ERR_CUDA", -4: "RT_ERR_TIMEOUT",
          -5: "RT_ERR_BOUNDS", -6: "RT_ERR_UNSUPPORTED", -7: "RT_ERR_STACK", -8: "RT_ERR_NO_DEVICE"}

KERNEL_MEGAKERNEL = 0
KERNEL_WAVEFRONT = 1

# Differentiable parameter vector (include/rt3d.h, RT_ADJ_*): 16 slots per
# material, then the medium's sigma_a[3], sigma_s[3].
ADJ_PER_MATERIAL = 16
ADJ_GLOBAL = 6
ADJ_SLOTS = {"base_color": 0, "radiance": 0, "roughness": 3, "metallic": 4, "specular": 5, "specular_tint": 6,
             "sheen": 7, "sheen_tint": 8, "clearcoat": 9, "spec_trans": 10, "anisotropic": 11, "absorption": 12}
ADJ_MEDIUM_SIGMA_A = 0
ADJ_MEDIUM_SIGMA_S = 3
ADJ_PARAMS_PER_MATERIAL = 12

F3 = C.c_float * 3


class RtMaterialDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("is_light_proxy", C.c_int32), ("thin_walled", C.c_int32),
                ("has_transmission_color", C.c_int32), ("base_color", F3), ("intensity", C.c_float),
                ("metallic", C.c_float), ("roughness", C.c_float), ("specular", C.c_float),
                ("specular_tint", C.c_float), ("sheen", C.c_float), ("sheen_tint", C.c_float),
                ("sheen_roughness", C.c_float), ("clearcoat", C.c_float), ("clearcoat_gloss", C.c_float),
                ("spec_trans", C.c_float), ("ior", C.c_float), ("anisotropic", C.c_float),
                ("anisotropic_rotation", C.c_float), ("diff_trans", C.c_float), ("coat_ior", C.c_float),
                ("coat_roughness", C.c_float), ("thin_film_thickness", C.c_float), ("thin_film_ior", C.c_float),
                ("transmission_color", F3), ("transmission_depth", C.c_float)]


class RtEntityDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("material", C.c_int32), ("flags", C.c_int32), ("pad", C.c_int32),
                ("first", C.c_int64), ("count", C.c_int64), ("p", C.c_float * 12)]


class RtLightDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("shadow_samples", C.c_int32), ("proxy_material", C.c_int32),
                ("pad", C.c_int32), ("corner", F3), ("u", F3), ("v", F3), ("color", F3),
                ("intensity", C.c_float), ("soft_radius", C.c_float), ("direction", F3),
                ("angular_radius_deg", C.c_float), ("center", F3), ("radius", C.c_float)]


class RtCameraDesc(C.Structure):
    _fields_ = [("look_from", F3), ("look_at", F3), ("vup", F3), ("vfov_deg", C.c_float),
                ("aperture", C.c_float), ("focus_dist", C.c_float)]


class RtMediumDesc(C.Structure):
    _fields_ = [("enabled", C.c_int32), ("pad", C.c_int32), ("sigma_a", F3), ("sigma_s", F3), ("g", C.c_float)]


class RtWorldDesc(C.Structure):
    _fields_ = [("materials", C.POINTER(RtMaterialDesc)), ("num_materials", C.c_int32),
                ("entities", C.POINTER(RtEntityDesc)), ("num_entities", C.c_int32),
                ("tri_verts", C.POINTER(C.c_float)), ("num_tris", C.c_int64),
                ("lights", C.POINTER(RtLightDesc)), ("num_lights", C.c_int32),
                ("geometry_light_samples", C.c_int32), ("camera", RtCameraDesc), ("medium", RtMediumDesc),
                ("tri_normals", C.POINTER(C.c_float)), ("tri_uvs", C.POINTER(C.c_float)),
                ("sky_color", F3), ("sky_light_samples", C.c_int32)]


class RtRenderParams(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("max_depth", C.c_int32),
                ("spp_offset", C.c_int32), ("rr_min_bounces", C.c_int32), ("rr_min_survival", C.c_float),
                ("max_sample_radiance", C.c_float), ("indirect_clamp_factor", C.c_float),
                ("exposure_ev", C.c_float), ("mis_heuristic", C.c_int32), ("light_strategy", C.c_int32),
                ("kernel", C.c_int32), ("block_size", C.c_int32), ("wavefront_size", C.c_int32),
                ("sort_materials", C.c_int32), ("pixel_x0", C.c_int32), ("pixel_y0", C.c_int32),
                ("window_w", C.c_int32), ("window_h", C.c_int32), ("count_work", C.c_int32), ("profile_kernels", C.c_int32),
                ("node_layout", C.c_int32), ("ray_fetch", C.c_int32), ("trace_block_size", C.c_int32),
                ("ray_groups", C.c_int32), ("iteration_limit", C.c_int32), ("shadow_queue_limit", C.c_int32)]


class RtStats(C.Structure):
    _fields_ = [("kernel_ms", C.c_double), ("total_ms", C.c_double), ("samples", C.c_uint64),
                ("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("node_visits", C.c_uint64),
                ("prim_tests", C.c_uint64), ("other_tests", C.c_uint64), ("shadow_node_visits", C.c_uint64),
                ("shadow_prim_tests", C.c_uint64), ("shadow_other_tests", C.c_uint64), ("regen_ms", C.c_double),
                ("extend_ms", C.c_double), ("shade_ms", C.c_double), ("occlude_ms", C.c_double),
                ("sort_ms", C.c_double), ("iterations", C.c_int32), ("kernel_launches", C.c_int32),
                ("rr_min_bounces", C.c_int32), ("rr_min_survival", C.c_float)]


class RtSceneInfo(C.Structure):
    _fields_ = [("num_nodes", C.c_int64), ("num_tris", C.c_int64), ("num_entities", C.c_int32),
                ("num_lights", C.c_int32), ("top_is_bvh", C.c_int32), ("max_stack_depth", C.c_int32),
                ("rr_min_bounces", C.c_int32), ("rr_min_survival", C.c_float), ("mean_irradiance", C.c_float),
                ("bvh_on_device", C.c_int32), ("device_bytes", C.c_int64), ("bvh_build_ms", C.c_double)]


BVH_AUTO, BVH_HOST, BVH_DEVICE = 0, 1, 2   # RT_BVH_*
BVH_AUTO_MIN_TRIS = 65536


class RtSceneOptions(C.Structure):
    _fields_ = [("bvh_build", C.c_int32), ("reserved", C.c_int32 * 7)]


class RtCapture(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("beauty_a", "beauty_b", "albedo_a", "albedo_b", "normal_a", "normal_b",
                                          "depth_a", "depth_b")]


class RtRequest(C.Structure):
    _fields_ = [("scene", C.c_int32), ("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32),
                ("max_depth", C.c_int32), ("pad", C.c_int32), ("camera", RtCameraDesc)]


class RtBsdfQuery(C.Structure):
    _fields_ = [("material", C.c_int32), ("front_face", C.c_int32), ("pixel_seed", C.c_uint32),
                ("sample_index", C.c_uint32), ("dim", C.c_uint32), ("pad", C.c_int32), ("n", F3),
                ("tangent", F3), ("bitangent", F3), ("v", F3), ("l", F3), ("point", F3)]


class RtBsdfResult(C.Structure):
    _fields_ = [("f", F3), ("pdf", C.c_float), ("fd", F3), ("pad0", C.c_float), ("wo", F3),
                ("s_pdf", C.c_float), ("s_f", F3), ("lobe", C.c_int32), ("is_delta", C.c_int32),
                ("has_sample", C.c_int32), ("dims_used", C.c_uint32), ("transition", C.c_int32)]


class RtMediumQuery(C.Structure):
    _fields_ = [("pixel_seed", C.c_uint32), ("sample_index", C.c_uint32), ("dim", C.c_uint32), ("tmax", C.c_float),
                ("wo", F3), ("wi", F3)]


class RtMediumResult(C.Structure):
    _fields_ = [("scattered", C.c_int32), ("dims_used", C.c_uint32), ("t", C.c_float), ("phase_eval", C.c_float),
                ("beta", F3), ("tr", F3), ("phase_wi", F3), ("phase_pdf", C.c_float)]


# numpy views of the two batch records (same layout as the C structs)
BSDF_QUERY_DTYPE = np.dtype([("material", "<i4"), ("front_face", "<i4"), ("pixel_seed", "<u4"),
                             ("sample_index", "<u4"), ("dim", "<u4"), ("pad", "<i4"), ("n", "<f4", 3),
                             ("tangent", "<f4", 3), ("bitangent", "<f4", 3), ("v", "<f4", 3),
                             ("l", "<f4", 3), ("point", "<f4", 3)])
BSDF_RESULT_DTYPE = np.dtype([("f", "<f4", 3), ("pdf", "<f4"), ("fd", "<f4", 3), ("pad0", "<f4"),
                              ("wo", "<f4", 3), ("s_pdf", "<f4"), ("s_f", "<f4", 3), ("lobe", "<i4"),
                              ("is_delta", "<i4"), ("has_sample", "<i4"), ("dims_used", "<u4"),
                              ("transition", "<i4")])
MEDIUM_QUERY_DTYPE = np.dtype([("pixel_seed", "<u4"), ("sample_index", "<u4"), ("dim", "<u4"), ("tmax", "<f4"),
                               ("wo", "<f4", 3), ("wi", "<f4", 3)])
MEDIUM_RESULT_DTYPE = np.dtype([("scattered", "<i4"), ("dims_used", "<u4"), ("t", "<f4"), ("phase_eval", "<f4"),
                                ("beta", "<f4", 3), ("tr", "<f4", 3), ("phase_wi", "<f4", 3),
                                ("phase_pdf", "<f4")])
assert BSDF_QUERY_DTYPE.itemsize == C.sizeof(RtBsdfQuery)
assert BSDF_RESULT_DTYPE.itemsize == C.sizeof(RtBsdfResult)
assert MEDIUM_QUERY_DTYPE.itemsize == C.sizeof(RtMediumQuery)
assert MEDIUM_RESULT_DTYPE.itemsize == C.sizeof(RtMediumResult)


def _f3(x):
    return F3(*[float(v) for v in x])


def camera_desc(c: dict) -> RtCameraDesc:
    return RtCameraDesc(_f3(c["look_from"]), _f3(c["look_at"]), _f3(c["vup"]), c["vfov"], c["aperture"],
                        c["focus_dist"])


class PackedWorld:
    """RtWorldDesc plus the buffers it points into (kept alive together)."""

    def __init__(self, world: "scenes.World"):
        nm = len(world.materials)
        self.mats = (RtMaterialDesc * max(nm, 1))()
        for i, m in enumerate(world.materials):
            d = self.mats[i]
            d.type = m["type"]
            d.is_light_proxy = int(bool(m["is_light_proxy"]))
            d.thin_walled = int(bool(m["thin_walled"]))
            d.has_transmission_color = int(m["transmission_color"] is not None)
            d.base_color = _f3(m["base_color"])
            d.intensity = m["intensity"]
            for k in ("metallic", "roughness", "specular", "specular_tint", "sheen", "sheen_tint",
                      "sheen_roughness", "clearcoat", "clearcoat_gloss", "spec_trans", "ior", "anisotropic",
                      "anisotropic_rotation", "diff_trans", "coat_ior", "coat_roughness", "thin_film_thickness",
                      "thin_film_ior", "transmission_depth"):
                setattr(d, k, float(m[k]))
            d.transmission_color = _f3(m["transmission_color"] or (1.0, 1.0, 1.0))
        ne = len(world.entities)
        self.ents = (RtEntityDesc * max(ne, 1))()
        for i, e in enumerate(world.entities):
            d = self.ents[i]
            d.kind = e["kind"]
            d.material = e["material"]
            d.flags = 1 if e.get("backface_culled") else 0
            p = [0.0] * 12
            if e["kind"] == scenes.ENT_QUAD:
                p[0:3], p[3:6], p[6:9] = e["q"], e["u"], e["v"]
            elif e["kind"] == scenes.ENT_SPHERE:
                p[0:3] = e["center"]
                p[3] = e["radius"]
            else:
                d.first, d.count = e["first"], e["count"]
            d.p = (C.c_float * 12)(*p)
        nl = len(world.lights)
        self.lights = (RtLightDesc * max(nl, 1))()
        for i, l in enumerate(world.lights):
            d = self.lights[i]
            d.type = l["type"]
            d.shadow_samples = int(l.get("shadow_samples", 0))
            d.proxy_material = int(l.get("proxy_material", -1))
            d.color = _f3(l["color"])
            d.intensity = l["intensity"]
            if l["type"] == scenes.LIGHT_AREA:
                d.corner, d.u, d.v = _f3(l["corner"]), _f3(l["u"]), _f3(l["v"])
                d.soft_radius = float(l.get("soft_radius", 0.0))
            elif l["type"] == scenes.LIGHT_SPHERE:
                d.center = _f3(l["center"])
                d.radius = float(l["radius"])
            else:
                d.direction = _f3(l["direction"])
                d.angular_radius_deg = float(l.get("angular_radius_deg", 0.0))
        self.tris = np.ascontiguousarray(world.tri_verts, np.float32).reshape(-1)
        med = RtMediumDesc()
        if world.medium:
            med.enabled = 1
            med.sigma_a = _f3(world.medium["sigma_a"])
            med.sigma_s = _f3(world.medium["sigma_s"])
            med.g = float(world.medium["g"])
        fp = C.POINTER(C.c_float)
        self.normals = self.uvs = None
        if getattr(world, "tri_normals", None) is not None:
            self.normals = np.ascontiguousarray(world.tri_normals, np.float32).reshape(-1)
            self.uvs = np.ascontiguousarray(world.tri_uvs, np.float32).reshape(-1)
            assert self.normals.size == 9 * world.num_tris and self.uvs.size == 6 * world.num_tris
        self.desc = RtWorldDesc(self.mats, nm, self.ents, ne,
                                self.tris.ctypes.data_as(fp), world.num_tris,
                                self.lights, nl, int(world.geometry_light_samples), camera_desc(world.camera), med,
                                self.normals.ctypes.data_as(fp) if self.normals is not None else fp(),
                                self.uvs.ctypes.data_as(fp) if self.uvs is not None else fp(),
                                _f3(getattr(world, "sky", (0.0, 0.0, 0.0))),
                                int(getattr(world, "sky_light_samples", 1)))

    def ref(self):
        return C.byref(self.desc)


def render_params(width, height, spp, max_depth, **kw) -> RtRenderParams:
    p = RtRenderParams()
    p.width, p.height, p.spp, p.max_depth = width, height, spp, max_depth
    p.rr_min_bounces = kw.pop("rr_min_bounces", -1)
    p.rr_min_survival = kw.pop("rr_min_survival", 0.0)
    p.max_sample_radiance = kw.pop("max_sample_radiance", 10.0)
    p.indirect_clamp_factor = kw.pop("indirect_clamp_factor", 0.25)
    p.sort_materials = kw.pop("sort_materials", -1)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class RtError(RuntimeError):
    pass


_lib = None


def load(path: str | None = None):
    """Loads librt3d.so (raises if it is missing: the product has no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RtError(f"librt3d.so not built at {p}; run __graft_entry__.build()")
    lib = C.CDLL(p)
    P = C.c_void_p
    sig = {
        "rt_abi_version": (C.c_int, []),
        "rt_checked_build": (C.c_int, []),
        "rt_last_error": (C.c_char_p, []),
        "rt_device_count": (C.c_int, []),
        "rt_scene_create": (C.c_int, [C.POINTER(RtWorldDesc), C.POINTER(P)]),
        "rt_scene_create_ex": (C.c_int, [C.POINTER(RtWorldDesc), C.POINTER(RtSceneOptions), C.POINTER(P)]),
        "rt_scene_destroy": (C.c_int, [P]),
        "rt_scene_info": (C.c_int, [P, C.POINTER(RtSceneInfo)]),
        "rt_scene_export_bvh": (C.c_int, [P, P, C.c_int64, P, C.c_int64, P, C.c_int64]),
        "rt_world_inspect": (C.c_int, [C.POINTER(RtWorldDesc), C.POINTER(RtSceneInfo), P, C.c_int64, P, C.c_int64,
                                       P, C.c_int64]),
        "rt_render": (C.c_int, [P, C.POINTER(RtRenderParams), P, C.POINTER(RtStats)]),
        "rt_render_device": (C.c_int, [P, C.POINTER(RtRenderParams), P, C.POINTER(RtStats)]),
        "rt_render_capture": (C.c_int, [P, C.POINTER(RtRenderParams), P, C.POINTER(RtCapture), C.POINTER(RtStats)]),
        "rt_render_device_noalloc": (C.c_int, [P, C.POINTER(RtRenderParams), P, C.POINTER(RtStats)]),
        "rt_render_batch": (C.c_int, [P, C.c_int32, P, C.c_int32, C.POINTER(RtRenderParams), P,
                                      C.POINTER(RtStats)]),
        "rt_adjoint": (C.c_int, [P, C.POINTER(RtRenderParams), P, P, P, C.c_int32, C.POINTER(RtStats)]),
        "rt_autotune": (C.c_int, [P, C.POINTER(RtRenderParams), C.POINTER(RtRenderParams)]),
        "rt_scene_get_params": (C.c_int, [P, P, C.c_int32]),
        "rt_scene_set_params": (C.c_int, [P, P, C.c_int32]),
        "rt_trace_closest": (C.c_int, [P, P, C.c_int64, C.c_float, C.c_float, P, C.c_int32]),
        "rt_trace_any": (C.c_int, [P, P, C.c_int64, P, C.c_int32]),
        "rt_bsdf_batch": (C.c_int, [P, P, C.c_int64, P]),
        "rt_medium_batch": (C.c_int, [P, P, C.c_int64, P]),
        "rt_sobol_batch": (C.c_int, [P, P, P, C.c_int64, P]),
        "rt_energy_lut": (C.c_int, [P, P]),
        "rt_probe_l2_bandwidth": (C.c_int, [C.c_int32, C.c_int64, C.c_int32, C.POINTER(C.c_double)]),
        "rt_tonemap": (C.c_int, [P, C.c_int32, C.c_int32, C.c_float, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib if path is None else _lib
    return lib


def check(rc: int, what: str = "rt call"):
    if rc != RT_OK:
        msg = load().rt_last_error()
        raise RtError(f"{what} failed: {ERRORS.get(rc, rc)}: {msg.decode() if msg else ''}")


def ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)
