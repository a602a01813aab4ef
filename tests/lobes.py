"""Inputs of the per-query BSDF and medium parity tests.

`lobe_world()` holds one Disney material for each part of the BSDF that the
Cornell and icosphere materials never reach (DisneyBsdf.cs ScatterInternal
:1176-1248 and its lobe samplers :1263-1709): the C4 sphere's sheen, the C5
glass (smooth and rough specular transmission, with total internal reflection
from inside), a thin-walled sheet, diffuse transmission, an anisotropic and
rotated GGX frame, a clearcoat below the delta threshold on both coat paths,
a rough metal whose multiscatter lobe is large, and one material that mixes
every lobe. `bsdf_queries()` draws shading inputs over them;
`medium_world()` and `medium_queries()` do the same for the homogeneous
medium and its Henyey-Greenstein phase.
"""
from __future__ import annotations

import numpy as np

from conftest import rt

abi = rt.abi
S = rt.scenes

LOBES = ("diffuse", "specular", "transmission", "sheen", "multiscatter", "difftrans", "clearcoat")

# name -> DisneyBsdf parameters (constructor defaults for the rest)
ZOO = {
    "c4_sheen": dict(color=(0.6, 0.3, 0.2), roughness=0.5, sheen=1.0, sheen_tint=0.5, sheen_roughness=0.3),
    "c5_glass": dict(color=(1.0, 1.0, 1.0), roughness=0.0, spec_trans=1.0, ior=1.5,
                     transmission_color=tuple(float(x) for x in np.exp(-np.array([0.1, 0.3, 0.5]))),
                     transmission_depth=1.0),
    "glass_rough": dict(color=(0.9, 0.95, 1.0), roughness=0.3, spec_trans=1.0, ior=1.5),
    "glass_rough_aniso": dict(color=(1.0, 1.0, 1.0), roughness=0.45, spec_trans=0.9, ior=1.33, anisotropic=0.6,
                              anisotropic_rotation=0.25),
    "thin_sheet": dict(color=(0.8, 0.9, 0.7), roughness=0.2, spec_trans=0.8, ior=1.4, thin_walled=True),
    "diff_trans": dict(color=(0.7, 0.6, 0.5), roughness=0.6, diff_trans=0.7),
    "aniso_metal": dict(color=(0.9, 0.7, 0.4), roughness=0.4, metallic=0.6, anisotropic=0.8,
                        anisotropic_rotation=0.3),
    "coat_gloss": dict(color=(0.2, 0.4, 0.8), roughness=0.5, clearcoat=1.0, clearcoat_gloss=0.4),
    "coat_rough": dict(color=(0.5, 0.1, 0.1), roughness=0.3, clearcoat=0.8, coat_roughness=0.2, coat_ior=1.6),
    "rough_metal": dict(color=(0.95, 0.8, 0.6), roughness=0.9, metallic=1.0),
    "everything": dict(color=(0.6, 0.6, 0.5), roughness=0.6, metallic=0.2, sheen=0.5, clearcoat=0.5,
                       clearcoat_gloss=0.7, spec_trans=0.3, diff_trans=0.3, anisotropic=0.5,
                       anisotropic_rotation=0.1, specular_tint=0.4),
}


def index(name: str) -> int:
    """Material index of a ZOO entry in lobe_world()."""
    return list(ZOO).index(name)


def lobe_world() -> "S.World":
    w = S.World(name="lobe-zoo")
    for name, p in ZOO.items():
        p = dict(p)
        color = p.pop("color")
        w.add_material(name, S.disney(color, **p))
    light = w.add_material("light", S.emissive((4.0, 4.0, 4.0), 1.0))
    for k in range(len(ZOO)):   # one small quad per material, so every material is in use
        w.add_quad((3.0 * k, 0, 0), (1, 0, 0), (0, 0, 1), k, name=f"quad{k}")
    w.add_quad((0, 5, 0), (1, 0, 0), (0, 0, 1), light, name="light")
    w.camera = S.camera((10.0, 3.0, -20.0), (10.0, 0.0, 0.0))
    return w


def _unit(rng, k):
    v = rng.normal(size=(k, 3)).astype(np.float32)
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def bsdf_queries(world, n: int, seed: int = 31, grazing: float = 0.1) -> np.ndarray:
    """n queries spread evenly over the world's Disney materials. The view
    direction is always on the normal's side (the renderer's face-forwarded
    normal), a `grazing` fraction of it within 3 degrees of the tangent
    plane; front_face is random, so transmissive materials are also entered
    from inside (eta = ior, total internal reflection); L for Evaluate/Pdf/
    EvaluateDirect covers both hemispheres."""
    rng = np.random.default_rng(seed)
    q = np.zeros(n, abi.BSDF_QUERY_DTYPE)
    disney = [i for i, m in enumerate(world.materials) if m["type"] == S.MAT_DISNEY]
    q["material"] = np.resize(np.array(disney, np.int32), n)
    rng.shuffle(q["material"])
    q["front_face"] = rng.integers(0, 2, n)
    q["pixel_seed"] = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    q["sample_index"] = rng.integers(0, 4096, n)
    q["dim"] = rng.integers(2, 40, n)
    nrm = _unit(rng, n)
    t = np.cross(nrm, _unit(rng, n)).astype(np.float32)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    b = np.cross(nrm, t).astype(np.float32)
    v = _unit(rng, n)
    v[np.sum(v * nrm, 1) < 0] *= -1
    g = rng.random(n) < grazing   # grazing views: cos between 0.001 and sin(3 deg)
    if np.any(g):
        cos = rng.uniform(1e-3, 0.052, int(g.sum())).astype(np.float32)
        tang = t[g] * np.cos(rng.uniform(0, 2 * np.pi, int(g.sum())))[:, None].astype(np.float32) + \
            b[g] * np.sin(rng.uniform(0, 2 * np.pi, int(g.sum())))[:, None].astype(np.float32)
        tang /= np.linalg.norm(tang, axis=1, keepdims=True)
        vv = tang * np.sqrt(1 - cos * cos)[:, None] + nrm[g] * cos[:, None]
        v[g] = (vv / np.linalg.norm(vv, axis=1, keepdims=True)).astype(np.float32)
    q["n"], q["tangent"], q["bitangent"], q["v"], q["l"] = nrm, t, b, v, _unit(rng, n)
    q["point"] = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    return q


# Henyey-Greenstein g values and media of the medium parity test: the C5 medium,
# a chromatic one with a vacuum channel (its hero draw takes no distance), a
# back-scattering one, and one below HG's isotropic threshold |g| < 1e-3.
MEDIA = {
    "c5": dict(sigma_a=(0.004,) * 3, sigma_s=(0.016,) * 3, g=0.6),
    "chromatic_vacuum_channel": dict(sigma_a=(0.05, 0.0, 0.01), sigma_s=(0.2, 0.0, 0.4), g=0.3),
    "backward": dict(sigma_a=(0.5, 0.2, 0.1), sigma_s=(1.0, 2.0, 0.5), g=-0.7),
    "isotropic": dict(sigma_a=(0.02, 0.03, 0.04), sigma_s=(0.1, 0.1, 0.1), g=5e-4),
    "forward_peaked": dict(sigma_a=(0.001, 0.001, 0.001), sigma_s=(0.01, 0.02, 0.03), g=0.95),
}


def medium_world(name: str) -> "S.World":
    w = S.cornell()
    w.name = f"medium-{name}"
    w.medium = dict(MEDIA[name])
    return w


def medium_queries(n: int, seed: int = 41) -> np.ndarray:
    """Segments from 0.01 to 1000 units (log-uniform) on random Sobol streams,
    with random phase directions."""
    rng = np.random.default_rng(seed)
    q = np.zeros(n, abi.MEDIUM_QUERY_DTYPE)
    q["pixel_seed"] = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    q["sample_index"] = rng.integers(0, 4096, n)
    q["dim"] = rng.integers(2, 60, n)
    q["tmax"] = np.exp(rng.uniform(np.log(0.01), np.log(1000.0), n)).astype(np.float32)
    q["wo"] = _unit(rng, n)
    q["wi"] = _unit(rng, n)
    return q
