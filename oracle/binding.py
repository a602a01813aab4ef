"""ctypes binding of the oracle (test infrastructure only).

The oracle is the CPU checker of the CUDA path: a C++ restatement of 3d-ray's
C# bounce loop (oracle/oracle.cpp). Only tests/, __graft_entry__.smoke() and
the cpu_baseline leg of bench.py import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P = C.c_void_p
        for name, res, args in [
            ("or_last_error", C.c_char_p, []),
            ("or_sobol", C.c_float, [C.c_uint32, C.c_uint32, C.c_uint32]),
            ("or_sobol_batch", C.c_int, [P, P, P, C.c_int64, P]),
            ("or_energy_lut", C.c_int, [P, P]),
            ("or_hg_eval", C.c_float, [C.c_float, P, P]),
            ("or_hg_sample", C.c_float, [C.c_float, P, C.c_float, C.c_float, P]),
            ("or_medium_transmittance", C.c_int, [P, C.c_float, P]),
            ("or_medium_sample", C.c_int, [P, P, C.c_float, C.c_float, C.c_float, P, P]),
            ("or_scene_create", C.c_int, [P, C.POINTER(P)]),
            ("or_scene_destroy", C.c_int, [P]),
            ("or_scene_info", C.c_int, [P, P, P, P, P, P]),
            ("or_export_top", C.c_int64, [P, P, C.c_int64, P, C.c_int64]),
            ("or_export_mesh", C.c_int64, [P, C.c_int32, P, C.c_int64, P, C.c_int64]),
            ("or_trace_closest", C.c_int, [P, P, C.c_int64, C.c_float, C.c_float, P, P, C.c_int32]),
            ("or_trace_any", C.c_int, [P, P, C.c_int64, P]),
            ("or_bsdf_batch", C.c_int, [P, P, C.c_int64, P]),
            ("or_medium_batch", C.c_int, [P, P, C.c_int64, P]),
            ("or_tonemap", C.c_int, [P, C.c_int32, C.c_int32, C.c_float, P]),
            ("or_render", C.c_int, [P, P, P, C.c_int32, P]),
            ("or_render_capture", C.c_int, [P, P, P, C.c_int32]),
        ]:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def sobol(idx, dim, seed) -> np.ndarray:
    idx = np.ascontiguousarray(idx, np.uint32)
    dim = np.ascontiguousarray(np.broadcast_to(dim, idx.shape), np.uint32)
    seed = np.ascontiguousarray(np.broadcast_to(seed, idx.shape), np.uint32)
    out = np.empty(idx.shape, np.float32)
    lib().or_sobol_batch(_p(idx), _p(dim), _p(seed), idx.size, _p(out))
    return out


def hg_eval(g, wo, wi) -> float:
    """HenyeyGreensteinPhase.Evaluate."""
    a = np.ascontiguousarray(wo, np.float32)
    b = np.ascontiguousarray(wi, np.float32)
    return float(lib().or_hg_eval(g, _p(a), _p(b)))


def hg_sample(g, wo, u1, u2):
    """HenyeyGreensteinPhase.Sample for the uniform draws (u1, u2): (wi, pdf)."""
    a = np.ascontiguousarray(wo, np.float32)
    wi = np.empty(3, np.float32)
    pdf = lib().or_hg_sample(g, _p(a), u1, u2, _p(wi))
    return wi, float(pdf)


def medium_transmittance(sigma_t, t) -> np.ndarray:
    s = np.ascontiguousarray(np.broadcast_to(np.asarray(sigma_t, np.float32), (3,)))
    out = np.empty(3, np.float32)
    lib().or_medium_transmittance(_p(s), t, _p(out))
    return out


def medium_sample(sigma_a, sigma_s, tmax, u_ch, u_d):
    """HomogeneousMedium.Sample for the draws (u_ch, u_d): (scattered, t, beta)."""
    sa = np.ascontiguousarray(np.broadcast_to(np.asarray(sigma_a, np.float32), (3,)))
    ss = np.ascontiguousarray(np.broadcast_to(np.asarray(sigma_s, np.float32), (3,)))
    t = np.zeros(1, np.float32)
    beta = np.empty(3, np.float32)
    sc = lib().or_medium_sample(_p(sa), _p(ss), tmax, u_ch, u_d, _p(t), _p(beta))
    return bool(sc), float(t[0]), beta


def tonemap(hdr_planar: np.ndarray, exposure_ev: float = 0.0) -> np.ndarray:
    """Renderer.ToneMapToDisplay with AcesToneMap: planar [3, H, W] HDR in,
    interleaved [H, W, 3] display RGB out."""
    hdr = np.ascontiguousarray(hdr_planar, np.float32)
    _, h, w = hdr.shape
    out = np.empty((h, w, 3), np.float32)
    rc = lib().or_tonemap(_p(hdr), w, h, exposure_ev, _p(out))
    if rc != 0:
        raise RuntimeError("oracle tonemap failed")
    return out


def energy_lut():
    e = np.empty(1024, np.float32)
    ea = np.empty(32, np.float32)
    lib().or_energy_lut(_p(e), _p(ea))
    return e, ea


class OracleScene:
    """A scene built by the oracle from the same RtWorldDesc the product takes."""

    def __init__(self, packed_world):
        self._packed = packed_world
        h = C.c_void_p()
        rc = lib().or_scene_create(C.cast(C.pointer(packed_world.desc), C.c_void_p), C.byref(h))
        if rc != 0:
            raise RuntimeError(f"oracle scene: {rc} {lib().or_last_error().decode()}")
        self.h = h

    def close(self):
        if self.h:
            lib().or_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        b = C.c_int32()
        s = C.c_float()
        m = C.c_float()
        n = C.c_int32()
        t = C.c_int32()
        lib().or_scene_info(self.h, C.byref(b), C.byref(s), C.byref(m), C.byref(n), C.byref(t))
        return dict(rr_min_bounces=b.value, rr_min_survival=s.value, mean_irradiance=m.value,
                    num_lights=n.value, top_is_bvh=t.value)

    def export_top(self):
        nodes = np.zeros((1 << 16, 10), np.int32)
        order = np.zeros(1 << 16, np.int32)
        n = lib().or_export_top(self.h, _p(nodes), nodes.shape[0], _p(order), order.size)
        return nodes[:n], order

    def export_mesh(self, entity: int, ntris: int):
        nodes = np.zeros((max(2 * ntris, 2), 10), np.int32)
        order = np.zeros(max(ntris, 1), np.int32)
        n = lib().or_export_mesh(self.h, entity, _p(nodes), nodes.shape[0], _p(order), order.size)
        return nodes[:max(n, 0)], order[:ntris]

    def trace_closest(self, rays: np.ndarray, tmin=1e-4, tmax=3.4028235e38, linear=False):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        hits = np.zeros((rays.shape[0], 6), np.int32)
        cnt = np.zeros(3, np.uint64)
        lib().or_trace_closest(self.h, _p(rays), rays.shape[0], tmin, tmax, _p(hits), _p(cnt), int(linear))
        return hits, cnt

    def trace_any(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        out = np.zeros((rays.shape[0], 3), np.float32)
        lib().or_trace_any(self.h, _p(rays), rays.shape[0], _p(out))
        return out

    def bsdf(self, queries: np.ndarray, result_dtype) -> np.ndarray:
        out = np.zeros(queries.shape[0], result_dtype)
        lib().or_bsdf_batch(self.h, _p(queries), queries.shape[0], _p(out))
        return out

    def medium(self, queries: np.ndarray, result_dtype) -> np.ndarray:
        """Medium and phase draws on each query's Sobol stream (RtMediumQuery
        records in, RtMediumResult records out)."""
        out = np.zeros(queries.shape[0], result_dtype)
        if lib().or_medium_batch(self.h, _p(queries), queries.shape[0], _p(out)) != 0:
            raise RuntimeError("oracle medium batch: the scene has no medium")
        return out

    def render_capture(self, params, threads: int | None = None) -> dict:
        """A capturing render of the whole frame: dict of beauty, beauty_a,
        beauty_b, albedo_a, albedo_b, normal_a, normal_b ([3, H, W]) and
        depth_a, depth_b ([H, W])."""
        W, H = params.width, params.height
        out = np.zeros((23, H, W), np.float32)
        nt = threads or os.cpu_count() or 1
        lib().or_render_capture(self.h, C.cast(C.pointer(params), C.c_void_p), _p(out), nt)
        names = ["beauty", "beauty_a", "beauty_b", "albedo_a", "albedo_b", "normal_a", "normal_b"]
        d = {n: out[3 * k:3 * k + 3] for k, n in enumerate(names)}
        d["depth_a"], d["depth_b"] = out[21], out[22]
        return d

    def render(self, params, threads: int | None = None, counters: bool = False):
        """Returns (planar [3,H,W] float32 film, counters dict or None)."""
        W, H = params.width, params.height
        out = np.zeros((3, H, W), np.float32)
        cnt = np.zeros(7, np.uint64)
        nt = threads or os.cpu_count() or 1
        lib().or_render(self.h, C.cast(C.pointer(params), C.c_void_p), _p(out), nt,
                        _p(cnt) if counters else None)
        c = None
        if counters:
            c = dict(zip(["node_visits", "tri_tests", "other_tests", "closest_rays", "shadow_rays", "segments",
                          "samples"], [int(x) for x in cnt]))
        return out, c
