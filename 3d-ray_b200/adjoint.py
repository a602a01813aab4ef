"""Differentiable rendering through the path-replay adjoint (rt_adjoint).

`DiffScene` holds a scene handle and its differentiable parameter vector: 16
slots per material, then the medium's sigma_a and sigma_s (slot names in
`abi.ADJ_SLOTS`). `render_function()` returns the torch.autograd.Function of
the gradient-check harness. Its forward renders the HDR film with rt_render for
a parameter vector. Its backward calls rt_adjoint, which re-traces the same
samples (same spp and spp_offset) and returns dLoss/dparams.

There is no counterpart in 3d-ray: the reference renders forward only.
"""
from __future__ import annotations

import copy
import ctypes as C

import numpy as np

from . import abi

# Parameter vectors up to this length gather their gradients in per-thread
# arrays inside the adjoint kernels; longer ones in shared memory.
ADJ_LOCAL_SLOTS = 128


class DiffScene:
    """A scene whose parameter vector can be read, written and differentiated."""

    def __init__(self, world):
        self.lib = abi.load()
        self._pw = abi.PackedWorld(world)
        self.handle = C.c_void_p()
        abi.check(self.lib.rt_scene_create(self._pw.ref(), C.byref(self.handle)), "rt_scene_create")
        self.num_materials = len(world.materials)
        self.count = self.num_materials * abi.ADJ_PER_MATERIAL + abi.ADJ_GLOBAL
        self.material_index = {name: i for i, name in enumerate(world.material_names)}
        self.last_stats = abi.RtStats()

    def slot(self, material: str | int, name: str, channel: int = 0) -> int:
        """Index of a material slot in the parameter vector."""
        m = self.material_index[material] if isinstance(material, str) else int(material)
        return m * abi.ADJ_PER_MATERIAL + abi.ADJ_SLOTS[name] + channel

    def medium_slot(self, name: str, channel: int = 0) -> int:
        base = self.num_materials * abi.ADJ_PER_MATERIAL
        return base + (abi.ADJ_MEDIUM_SIGMA_A if name == "sigma_a" else abi.ADJ_MEDIUM_SIGMA_S) + channel

    def medium_albedo_direction(self, theta, channel: int = 0) -> dict:
        """The medium's single-scattering albedo a = sigma_s / sigma_t of one
        channel as a direction in the parameter vector at a fixed sigma_t:
        d sigma_s / da = sigma_t, d sigma_a / da = -sigma_t. Returns {slot:
        coefficient}; dLoss/da is the sum of coefficient * dLoss/dslot."""
        ia, isc = self.medium_slot("sigma_a", channel), self.medium_slot("sigma_s", channel)
        st = float(theta[ia]) + float(theta[isc])
        return {isc: st, ia: -st}

    def medium_albedo_gradient(self, theta, grad, channel: int = 0) -> float:
        """dLoss/d(albedo) of one channel at a fixed sigma_t, from the gradient
        rt_adjoint returns for the sigma_a and sigma_s slots."""
        return float(sum(c * float(grad[i]) for i, c in self.medium_albedo_direction(theta, channel).items()))

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.count, np.float32)
        abi.check(self.lib.rt_scene_get_params(self.handle, abi.ptr(out), self.count), "rt_scene_get_params")
        return out

    def set_params(self, params) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.shape != (self.count,):
            raise ValueError(f"parameter vector must have {self.count} entries")
        abi.check(self.lib.rt_scene_set_params(self.handle, abi.ptr(p), self.count), "rt_scene_set_params")

    def render(self, params: abi.RtRenderParams) -> np.ndarray:
        film = np.zeros((3, params.height, params.width), np.float32)
        st = abi.RtStats()
        abi.check(self.lib.rt_render(self.handle, C.byref(params), abi.ptr(film), C.byref(st)), "rt_render")
        return film

    def adjoint(self, params: abi.RtRenderParams, d_image: np.ndarray, mask=None) -> np.ndarray:
        """dLoss/dparams for dLoss/dfilm = d_image (3 x H x W, linear HDR).
        mask: the slots to differentiate (bool array or index list); None = all."""
        g = np.ascontiguousarray(d_image, dtype=np.float32)
        if g.shape != (3, params.height, params.width):
            raise ValueError("d_image must be 3 x H x W")
        mp = None
        if mask is not None:
            m = np.zeros(self.count, np.uint8)
            mk = np.asarray(mask)
            if mk.dtype == bool:
                m[:] = mk
            else:
                m[mk.astype(int)] = 1
            self._mask = m
            mp = abi.ptr(m)
        out = np.zeros(self.count, np.float32)
        self.last_stats = abi.RtStats()
        abi.check(self.lib.rt_adjoint(self.handle, C.byref(params), abi.ptr(g), mp, abi.ptr(out), self.count,
                                      C.byref(self.last_stats)), "rt_adjoint")
        return out

    def close(self):
        if self.handle:
            self.lib.rt_scene_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_DISNEY_SLOTS = ["roughness", "metallic", "specular", "specular_tint", "sheen", "sheen_tint", "clearcoat", "spec_trans",
                 "anisotropic"]


def world_with_params(world, params, reference=None):
    """A copy of `world` with the parameter vector applied the way
    rt_scene_set_params applies it, for renderers that take a world
    description (the CPU oracle). `reference` is the vector the world
    currently has (DiffScene.get_params()); slots equal to it are left alone,
    as the library does."""
    w = copy.deepcopy(world)
    p = np.asarray(params, np.float32)
    ref = None if reference is None else np.asarray(reference, np.float32)
    per = abi.ADJ_PER_MATERIAL
    ab = abi.ADJ_SLOTS["absorption"]
    for i, m in enumerate(w.materials):
        q = p[i * per:(i + 1) * per]
        r = None if ref is None else ref[i * per:(i + 1) * per]
        if m["type"] == 1:   # Emissive: radiance = colour * intensity
            if r is not None and np.array_equal(q[:3], r[:3]):
                continue
            if not m["intensity"] > 0.0:
                m["intensity"] = 1.0
            col = list(m["base_color"])
            for c in range(3):
                if r is None or q[c] != r[c]:
                    col[c] = float(np.float32(q[c]) / np.float32(m["intensity"]))
            m["base_color"] = tuple(col)
            continue
        m["base_color"] = tuple(float(x) for x in q[0:3])
        for k, name in enumerate(_DISNEY_SLOTS):
            m[name] = float(q[3 + k])
        sg = q[ab:ab + 3]
        if r is not None and np.array_equal(sg, r[ab:ab + 3]):
            continue
        has_depth = m.get("transmission_color") is not None and m.get("transmission_depth", 0.0) > 0.0
        if r is None and not has_depth and not np.any(sg):
            continue
        if not has_depth:
            m["transmission_depth"] = 1.0
        depth = np.float32(m["transmission_depth"])
        m["transmission_color"] = tuple(float(np.exp(-np.maximum(np.float32(x), 0) * depth)) for x in sg)
    if w.medium is not None:
        g = p[len(w.materials) * per:]
        w.medium = dict(w.medium)
        w.medium["sigma_a"] = tuple(float(x) for x in g[abi.ADJ_MEDIUM_SIGMA_A:abi.ADJ_MEDIUM_SIGMA_A + 3])
        w.medium["sigma_s"] = tuple(float(x) for x in g[abi.ADJ_MEDIUM_SIGMA_S:abi.ADJ_MEDIUM_SIGMA_S + 3])
    return w


def render_function():
    """Returns the torch.autograd.Function class (torch is imported lazily)."""
    import torch

    class RenderFunction(torch.autograd.Function):
        """image = render(theta). The backward pass replays the forward's
        samples, so the scene must keep theta until backward runs."""

        @staticmethod
        def forward(ctx, theta, scene: DiffScene, params: abi.RtRenderParams, mask=None):
            scene.set_params(theta.detach().cpu().numpy())
            ctx.scene = scene
            ctx.params = params
            ctx.mask = mask
            return torch.from_numpy(scene.render(params))

        @staticmethod
        def backward(ctx, grad_image):
            g = ctx.scene.adjoint(ctx.params, grad_image.detach().cpu().numpy(), ctx.mask)
            return torch.from_numpy(g), None, None, None

    return RenderFunction
