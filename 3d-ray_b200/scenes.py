"""Synthetic scene generators for the path-tracing core.

There is no public dataset behind the reference's benchmark configurations, so
every scene is generated from a seed (PCG64 via numpy). A scene is returned as
an entity-level `World` — the same information 3d-ray's YAML loader produces
(materials, entities in YAML order, explicit lights, camera, optional global
medium) — which `abi.pack_world` turns into the C-ABI `RtWorldDesc`.
`write_yaml` writes the same world as reference-compatible YAML + OBJ so that
anyone with .NET can render identical inputs with the C# renderer.

Configurations (sizes from the reference's benchmark text):
  cornell()            C1: 555-unit Cornell box, 5 wall quads, 2 rotated
                       12-triangle boxes, one 130x105 emissive ceiling quad.
  throughput_scene()   C2: 64 fBm-displaced icospheres (level 5, 20 480
                       triangles each; 16 384 is not an icosphere level) on a
                       2-triangle ground, 64 random Disney materials, one area
                       light (with its back-face-culled proxy quad) + a sun.
  cornell_sphere()     C4: C1 plus a Disney sphere of radius 80.
  cornell_volume()     C5: C1 with a homogeneous medium and a dielectric sphere
                       replacing the tall box.
  batch_requests()     C3: 32 uneven render requests over C1 / C2.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Any

import numpy as np

MAT_DISNEY = 0
MAT_EMISSIVE = 1
ENT_QUAD = 0
ENT_SPHERE = 1
ENT_MESH = 2
LIGHT_AREA = 0
LIGHT_DIRECTIONAL = 1
LIGHT_SPHERE = 2

DEFAULT_SCENE_SEED = 0x3D7A1
DEFAULT_REQUEST_SEED = 0xC0FFEE


def disney(color, **kw) -> dict:
    """A Disney material with the DisneyBsdf constructor defaults
    (src/RayTracer/Materials/DisneyBsdf.cs:195-215)."""
    m = dict(type=MAT_DISNEY, base_color=tuple(float(c) for c in color), metallic=0.0, roughness=0.5,
             specular=0.5, specular_tint=0.0, sheen=0.0, sheen_tint=0.5, sheen_roughness=0.3, clearcoat=0.0,
             clearcoat_gloss=1.0, spec_trans=0.0, ior=1.5, anisotropic=0.0, anisotropic_rotation=0.0,
             diff_trans=0.0, coat_ior=1.5, coat_roughness=-1.0, thin_film_thickness=0.0, thin_film_ior=1.5,
             transmission_color=None, transmission_depth=0.0, thin_walled=False, intensity=0.0,
             is_light_proxy=False)
    m.update(kw)
    return m


def emissive(color, intensity=1.0, is_light_proxy=False) -> dict:
    m = disney(color)
    m.update(type=MAT_EMISSIVE, intensity=float(intensity), is_light_proxy=is_light_proxy)
    return m


@dataclasses.dataclass
class World:
    materials: list = dataclasses.field(default_factory=list)
    material_names: list = dataclasses.field(default_factory=list)
    entities: list = dataclasses.field(default_factory=list)
    tri_verts: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros((0, 9), np.float32))
    # smooth triangles (SmoothTriangle): per triangle n0, n1, n2 (zeros for a
    # flat one) and uv0, uv1, uv2; None while no triangle is smooth
    tri_normals: np.ndarray | None = None
    tri_uvs: np.ndarray | None = None
    lights: list = dataclasses.field(default_factory=list)
    geometry_light_samples: int = 1
    sky: tuple = (0.0, 0.0, 0.0)      # flat sky radiance (FlatSky); black: no EnvironmentLight
    sky_light_samples: int = 1        # the EnvironmentLight's ShadowSamples
    camera: dict = dataclasses.field(default_factory=dict)
    medium: dict | None = None
    name: str = ""

    # -- building helpers ---------------------------------------------------
    def add_material(self, name: str, m: dict) -> int:
        self.materials.append(m)
        self.material_names.append(name)
        return len(self.materials) - 1

    def add_quad(self, q, u, v, material: int, backface_culled=False, name=""):
        self.entities.append(dict(kind=ENT_QUAD, material=material, q=tuple(map(float, q)),
                                  u=tuple(map(float, u)), v=tuple(map(float, v)),
                                  backface_culled=backface_culled, name=name))

    def add_sphere(self, center, radius, material: int, name=""):
        self.entities.append(dict(kind=ENT_SPHERE, material=material, center=tuple(map(float, center)),
                                  radius=float(radius), name=name))

    def add_sphere_light(self, center, radius, color, intensity, shadow_samples=4, name=""):
        """A SphereLight with its visible emissive proxy sphere, appended to the
        objects as SceneLoader.CreateSphereLight does (SceneLoader.cs:3592-3634)."""
        proxy = self.add_material(f"{name or 'sphere_light'}_proxy",
                                  emissive(color, intensity, is_light_proxy=True))
        self.add_sphere(center, radius, proxy, name=f"{name or 'sphere_light'}_proxy")
        self.lights.append(dict(type=LIGHT_SPHERE, center=tuple(map(float, center)), radius=float(radius),
                                color=tuple(map(float, color)), intensity=float(intensity),
                                shadow_samples=int(shadow_samples), proxy_material=proxy))

    def add_mesh(self, tris: np.ndarray, material: int, name="", normals=None, uvs=None, path=None):
        """A mesh entity of world-space triangles [n, 9]. With `normals`
        ([n, 9] vertex normals) its triangles are smooth, with `uvs` ([n, 6])
        their tangent frame follows the UV mapping; `path` records the OBJ the
        triangles came from."""
        tris = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
        n = tris.shape[0]
        first = self.tri_verts.shape[0]
        self.tri_verts = np.concatenate([self.tri_verts, tris], 0) if first else tris.copy()
        if normals is not None or self.tri_normals is not None:
            nn = np.zeros((n, 9), np.float32) if normals is None else \
                np.ascontiguousarray(normals, np.float32).reshape(n, 9)
            uu = np.tile(np.array([0, 0, 1, 0, 0, 1], np.float32), (n, 1)) if uvs is None else \
                np.ascontiguousarray(uvs, np.float32).reshape(n, 6)
            if self.tri_normals is None:
                self.tri_normals = np.zeros((first, 9), np.float32)
                self.tri_uvs = np.tile(np.array([0, 0, 1, 0, 0, 1], np.float32), (first, 1))
            self.tri_normals = np.concatenate([self.tri_normals, nn], 0)
            self.tri_uvs = np.concatenate([self.tri_uvs, uu], 0)
        self.entities.append(dict(kind=ENT_MESH, material=material, first=first, count=n, name=name,
                                  path=path))

    def add_obj(self, path: str, material: int, name=""):
        """A mesh entity loaded from an OBJ file the way the reference's
        ObjLoader does without subdivision (see objfile.load_obj); returns the
        loader's warnings."""
        from . import objfile
        m = objfile.load_obj(path)
        self.add_mesh(m.tris, material, name=name or os.path.basename(path), normals=m.normals, uvs=m.uvs,
                      path=path)
        return m.warnings

    @property
    def num_tris(self) -> int:
        return int(self.tri_verts.shape[0])

    def with_camera(self, **cam) -> "World":
        w = dataclasses.replace(self)
        w.camera = dict(self.camera)
        w.camera.update(cam)
        return w


def camera(look_from, look_at, vup=(0, 1, 0), vfov=40.0, aperture=0.0, focus_dist=1.0) -> dict:
    return dict(look_from=tuple(map(float, look_from)), look_at=tuple(map(float, look_at)),
                vup=tuple(map(float, vup)), vfov=float(vfov), aperture=float(aperture),
                focus_dist=float(focus_dist))


# --- geometry helpers --------------------------------------------------------

def box_triangles(size, rot_y_deg, translate) -> np.ndarray:
    """12 triangles of an axis-aligned box [0,size] rotated about y through its
    corner, then translated (the RTOW Cornell construction). Faces are wound
    outward; triangle winding only affects which side reads as front."""
    sx, sy, sz = size
    c = np.array([[0, 0, 0], [sx, 0, 0], [sx, sy, 0], [0, sy, 0],
                  [0, 0, sz], [sx, 0, sz], [sx, sy, sz], [0, sy, sz]], np.float64)
    faces = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (3, 7, 6, 2), (0, 4, 7, 3), (1, 2, 6, 5)]
    a = math.radians(rot_y_deg)
    ca, sa = math.cos(a), math.sin(a)
    rot = np.array([[ca, 0, sa], [0, 1, 0], [-sa, 0, ca]])
    p = c @ rot.T + np.asarray(translate, np.float64)
    tris = []
    for f in faces:
        tris.append(np.concatenate([p[f[0]], p[f[1]], p[f[2]]]))
        tris.append(np.concatenate([p[f[0]], p[f[2]], p[f[3]]]))
    return np.asarray(tris, np.float32)


def icosphere(level: int):
    """Unit icosphere by repeated 4:1 subdivision: 20*4**level triangles."""
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = np.asarray(verts, np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.asarray(faces, np.int64)
    for _ in range(level):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], 0)
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        mids = v[uniq[:, 0]] + v[uniq[:, 1]]
        mids /= np.linalg.norm(mids, axis=1, keepdims=True)
        base = v.shape[0]
        v = np.concatenate([v, mids], 0)
        n = f.shape[0]
        m01, m12, m20 = (inv[:n] + base, inv[n:2 * n] + base, inv[2 * n:] + base)
        f = np.concatenate([np.stack([f[:, 0], m01, m20], 1), np.stack([f[:, 1], m12, m01], 1),
                            np.stack([f[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)], 0)
    return v, f


def _hash3(ix, iy, iz, seed):
    h = (ix * 0x8DA6B343 + iy * 0xD8163841 + iz * 0xCB1AB31F + seed * 0x165667B1) & 0xFFFFFFFF
    h ^= h >> 13
    h = (h * 0x5BD1E995) & 0xFFFFFFFF
    h ^= h >> 15
    return h.astype(np.float64) / 4294967295.0 * 2.0 - 1.0


def value_noise(p: np.ndarray, seed: int) -> np.ndarray:
    """Smooth 3-D lattice value noise in [-1, 1] (trilinear over quintic fades)."""
    fl = np.floor(p)
    i = fl.astype(np.int64)
    f = p - fl
    w = f * f * f * (f * (f * 6 - 15) + 10)
    out = np.zeros(p.shape[0])
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                g = _hash3(i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz, seed)
                wx = w[:, 0] if dx else 1 - w[:, 0]
                wy = w[:, 1] if dy else 1 - w[:, 1]
                wz = w[:, 2] if dz else 1 - w[:, 2]
                out += g * wx * wy * wz
    return out


def fbm(p: np.ndarray, seed: int, octaves=4, lacunarity=2.0, gain=0.5) -> np.ndarray:
    total, amp, freq, norm = np.zeros(p.shape[0]), 1.0, 1.0, 0.0
    for o in range(octaves):
        total += amp * value_noise(p * freq, seed + 131 * o)
        norm += amp
        amp *= gain
        freq *= lacunarity
    return total / norm


# --- configurations ----------------------------------------------------------

def cornell(shadow_samples: int = 1, tall_box: bool = True) -> World:
    """C1. Camera looks down +z from z=-800; screen-left is +x (red wall)."""
    w = World(name="cornell-256")
    white = w.add_material("white", disney((0.73, 0.73, 0.73), roughness=1.0, metallic=0.0, specular=0.5))
    red = w.add_material("red", disney((0.65, 0.05, 0.05), roughness=1.0, metallic=0.0, specular=0.5))
    green = w.add_material("green", disney((0.12, 0.45, 0.15), roughness=1.0, metallic=0.0, specular=0.5))
    light = w.add_material("light", emissive((17.0, 12.0, 4.0), 1.0))
    w.add_quad((0, 0, 0), (555, 0, 0), (0, 0, 555), white, name="floor")
    w.add_quad((555, 555, 555), (-555, 0, 0), (0, 0, -555), white, name="ceiling")
    w.add_quad((0, 0, 555), (555, 0, 0), (0, 555, 0), white, name="back")
    w.add_quad((555, 0, 0), (0, 555, 0), (0, 0, 555), red, name="left")
    w.add_quad((0, 0, 0), (0, 555, 0), (0, 0, 555), green, name="right")
    # 130 x 105 emitter just under the ceiling; U x V points down (-y).
    w.add_quad((213, 554, 227), (130, 0, 0), (0, 0, 105), light, name="ceiling_light")
    w.add_mesh(box_triangles((165, 165, 165), -18.0, (130, 0, 65)), white, name="short_box")
    if tall_box:
        w.add_mesh(box_triangles((165, 330, 165), 18.0, (265, 0, 295)), white, name="tall_box")
    w.geometry_light_samples = shadow_samples
    w.camera = camera((278, 278, -800), (278, 278, 0), (0, 1, 0), 40.0)
    return w


def cornell_sphere(params: dict | None = None, shadow_samples: int = 1) -> World:
    """C4: C1 plus a Disney sphere (r = 80) whose parameters are fitted."""
    w = cornell(shadow_samples)
    w.name = "cornell-sphere"
    p = dict(base_color=(0.5, 0.5, 0.5), roughness=0.5, metallic=0.0, specular=0.5, sheen=0.0)
    if params:
        p.update(params)
    m = w.add_material("fit_sphere", disney(p["base_color"], roughness=p["roughness"], metallic=p["metallic"],
                                            specular=p["specular"], sheen=p["sheen"]))
    w.add_sphere((380, 80, 140), 80.0, m, name="fit_sphere")
    return w


def smooth_icosphere(level: int, center, radius: float, with_uvs: bool = True):
    """Triangles [n, 9] of a level-`level` icosphere of `radius` around
    `center`, its exact vertex normals [n, 9] (smooth triangles) and, with
    `with_uvs`, a longitude/latitude mapping [n, 6] (else None)."""
    v, f = icosphere(level)
    tris = (v * float(radius) + np.asarray(center, np.float64))[f].reshape(-1, 9).astype(np.float32)
    normals = v[f].reshape(-1, 9).astype(np.float32)
    uvs = None
    if with_uvs:
        lon = np.arctan2(v[:, 2], v[:, 0]) / (2 * math.pi) + 0.5
        lat = np.arcsin(np.clip(v[:, 1], -1, 1)) / math.pi + 0.5
        uvs = np.stack([lon, lat], 1)[f].reshape(-1, 6).astype(np.float32)
    return tris, normals, uvs


def cornell_smooth(shadow_samples: int = 1) -> World:
    """Smooth triangles (SmoothTriangle) in the Cornell box: a UV-mapped
    smooth icosphere with an anisotropic metallic Disney material in place of
    the tall box (its shading normal and UV tangent frame both matter) and a
    small smooth emissive icosphere, a geometry light whose samples and pdf
    use the interpolated normal."""
    w = cornell(shadow_samples, tall_box=False)
    w.name = "cornell-smooth"
    aniso = w.add_material("aniso", disney((0.8, 0.6, 0.3), roughness=0.3, metallic=0.7, anisotropic=0.8))
    tris, nn, uv = smooth_icosphere(3, (370, 100, 350), 100.0)
    w.add_mesh(tris, aniso, name="smooth_sphere", normals=nn, uvs=uv)
    glow = w.add_material("glow", emissive((6.0, 5.0, 3.0), 1.0))
    tris, nn, _ = smooth_icosphere(1, (150, 380, 300), 35.0, with_uvs=False)
    w.add_mesh(tris, glow, name="smooth_light", normals=nn)
    return w


def cornell_spheres(shadow_samples: int = 1) -> World:
    """Spherical emitters in the Cornell box: an emissive sphere (a
    GeometryLight sampled in its solid-angle cone) beside the ceiling quad,
    and a SphereLight with its proxy, both seen directly and through a
    metallic sphere."""
    w = cornell(shadow_samples, tall_box=False)
    w.name = "cornell-spheres"
    glow = w.add_material("glow_sphere", emissive((8.0, 6.0, 2.0), 1.0))
    w.add_sphere((140, 420, 350), 40.0, glow, name="glow_sphere")
    metal = w.add_material("metal", disney((0.9, 0.9, 0.9), roughness=0.25, metallic=1.0))
    w.add_sphere((380, 100, 380), 100.0, metal, name="metal_sphere")
    w.add_sphere_light((420, 330, 200), 25.0, (1.0, 0.8, 0.6), 12.0, shadow_samples=4, name="bulb")
    return w


def sky_scene(sky=(0.35, 0.45, 0.65)) -> World:
    """An open scene under a flat sky (FlatSky + EnvironmentLight): a ground
    quad, a glossy and a diffuse sphere and a glass sphere with interior
    absorption, with the camera seeing the sky above the horizon."""
    w = World(name="sky")
    ground = w.add_material("ground", disney((0.6, 0.6, 0.55), roughness=0.9))
    red = w.add_material("red", disney((0.7, 0.15, 0.1), roughness=0.6))
    gloss = w.add_material("gloss", disney((0.9, 0.9, 0.9), roughness=0.15, metallic=1.0))
    glass = w.add_material("glass", disney((1.0, 1.0, 1.0), roughness=0.0, spec_trans=1.0, ior=1.5,
                                           transmission_color=(0.6, 0.8, 0.9), transmission_depth=1.0))
    w.add_quad((-50, 0, -50), (100, 0, 0), (0, 0, 100), ground, name="ground")
    w.add_sphere((-2.2, 1.0, 0.0), 1.0, red, name="red")
    w.add_sphere((0.0, 1.0, 1.5), 1.0, gloss, name="gloss")
    w.add_sphere((2.2, 1.0, 0.0), 1.0, glass, name="glass")
    w.sky = tuple(float(x) for x in sky)
    w.camera = camera((0.0, 2.5, -7.0), (0.0, 1.0, 0.0), (0, 1, 0), 45.0)
    return w


def cornell_volume(shadow_samples: int = 1, density: float = 1.0) -> World:
    """C5: homogeneous medium (sigma_t 0.02 per unit times `density`, albedo
    0.8, HG g 0.6) filling the box, and a dielectric sphere (IOR 1.5,
    Beer-Lambert sigma_a (0.1,0.3,0.5) per unit via transmission_color =
    exp(-sigma_a), depth 1) in place of the tall box. The medium is global, so
    the camera sits in the box's open side (at sigma_t 0.02 the 800 units from
    the C1 camera alone have optical depth 16)."""
    w = cornell(shadow_samples, tall_box=False)
    w.name = "cornell-volume"
    sig = np.array([0.1, 0.3, 0.5])
    glass = w.add_material("glass", disney((1.0, 1.0, 1.0), roughness=0.0, spec_trans=1.0, ior=1.5,
                                           transmission_color=tuple(float(x) for x in np.exp(-sig)),
                                           transmission_depth=1.0))
    w.add_sphere((370, 90, 350), 90.0, glass, name="glass_sphere")
    w.medium = dict(sigma_a=(0.004 * density,) * 3, sigma_s=(0.016 * density,) * 3, g=0.6)
    w.camera = camera((278, 278, 1), (278, 278, 555), (0, 1, 0), 75.0)
    return w


def volume_views(n: int = 8) -> list:
    """C5's eight views: cameras on a circle of radius 80 in the box's open
    side, all looking at the box centre."""
    views = []
    for k in range(n):
        a = 2.0 * math.pi * k / n
        eye = (278.0 + 80.0 * math.cos(a), 278.0 + 80.0 * math.sin(a), 1.0)
        views.append(camera(eye, (278, 278, 278), (0, 1, 0), 75.0))
    return views


def throughput_scene(seed: int = DEFAULT_SCENE_SEED, n_spheres: int = 64, level: int = 5,
                     shadow_samples: int = 1) -> World:
    """C2: ~1.31 M triangles (64 x 20 480 + 2)."""
    rng = np.random.default_rng(seed)
    w = World(name=f"icospheres-{n_spheres}x{20 * 4 ** level}")
    unit_v, faces = icosphere(level)
    mats = []
    for k in range(n_spheres):
        mats.append(w.add_material(
            f"sphere_{k}",
            disney(tuple(rng.uniform(0.0, 1.0, 3)), roughness=float(rng.uniform(0.05, 1.0)),
                   metallic=1.0 if rng.uniform() < 0.3 else 0.0, specular=0.5,
                   clearcoat=float(rng.uniform(0.0, 1.0)))))
    ground = w.add_material("ground", disney((0.6, 0.6, 0.6), roughness=0.8))
    proxy = w.add_material("area_light_proxy", emissive((1.0, 0.95, 0.9), 6.0, is_light_proxy=True))
    centers = rng.uniform(-10.0, 10.0, (n_spheres, 3))
    radii = rng.uniform(0.3, 1.5, n_spheres)
    for k in range(n_spheres):
        disp = fbm(unit_v * 2.0 + centers[k], seed + k)
        v = unit_v * (radii[k] * (1.0 + 0.05 * disp))[:, None] + centers[k]
        tris = v[faces].reshape(-1, 9).astype(np.float32)
        w.add_mesh(tris, mats[k], name=f"icosphere_{k}")
    g = 20.0
    y = -11.5
    ground_tris = np.array([[-g, y, -g, g, y, -g, g, y, g], [-g, y, -g, g, y, g, -g, y, g]], np.float32)
    w.add_mesh(ground_tris, ground, name="ground")
    corner, u, v = (-5.0, 14.0, -5.0), (10.0, 0.0, 0.0), (0.0, 0.0, 10.0)
    # Area light: its visible proxy quad is appended to the objects after the
    # entities (SceneLoader.CreateAreaLight, src/RayTracer/Scene/SceneLoader.cs:3576-3585).
    w.add_quad(corner, u, v, proxy, backface_culled=True, name="area_light_proxy")
    w.lights.append(dict(type=LIGHT_AREA, corner=corner, u=u, v=v, color=(1.0, 0.95, 0.9), intensity=6.0,
                         shadow_samples=shadow_samples, proxy_material=proxy, soft_radius=0.0))
    w.lights.append(dict(type=LIGHT_DIRECTIONAL, direction=(-1.0, -2.0, -1.0), color=(1.0, 0.98, 0.92),
                         intensity=2.0, shadow_samples=shadow_samples, angular_radius_deg=0.0))
    w.geometry_light_samples = shadow_samples
    w.camera = camera((0.0, 6.0, -34.0), (0.0, -1.0, 0.0), (0, 1, 0), 40.0)
    return w


def batch_requests(n: int = 32, seed: int = DEFAULT_REQUEST_SEED, radius: float = 25.0):
    """C3 requests: scene Bernoulli(0.5) over {0: throughput scene, 1: Cornell},
    square resolution log-uniform in [64, 1024] snapped to multiples of 8, spp
    log-uniform in [16, 256], depth uniform in {4..12}, camera on a sphere of
    `radius` (scaled by the scene radius for the Cornell box) looking at the
    scene centre."""
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(n):
        scene = int(rng.uniform() < 0.5)
        res = int(round(math.exp(rng.uniform(math.log(64), math.log(1024))) / 8.0)) * 8
        spp = int(round(math.exp(rng.uniform(math.log(16), math.log(256)))))
        depth = int(rng.integers(4, 13))
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        if scene == 1:   # Cornell: stay inside the open front half-space
            center = np.array([278.0, 278.0, 278.0])
            d[2] = -abs(d[2]) - 0.5
            d /= np.linalg.norm(d)
            r = radius * 40.0
        else:
            center = np.array([0.0, -1.0, 0.0])
            d[1] = abs(d[1]) * 0.6 + 0.1
            d /= np.linalg.norm(d)
            r = radius
        eye = center + d * r
        reqs.append(dict(scene=scene, width=res, height=res, spp=spp, max_depth=depth,
                         camera=camera(tuple(eye), tuple(center), (0, 1, 0), 40.0)))
    return reqs


# --- reference-compatible YAML + OBJ ------------------------------------------

def write_yaml(world: World, out_dir: str, name: str | None = None) -> str:
    """Writes `<name>.yaml` plus one OBJ per mesh entity (world-space vertices;
    smooth meshes with their vertex normals and UVs, which ObjLoader turns into
    SmoothTriangle faces, flat ones without, which it turns into Triangle)."""
    import yaml

    name = name or world.name or "scene"
    os.makedirs(out_dir, exist_ok=True)
    mats = []
    for nm, m in zip(world.material_names, world.materials):
        if m["is_light_proxy"]:
            continue
        if m["type"] == MAT_EMISSIVE:
            mats.append(dict(id=nm, type="emissive", color=list(m["base_color"]), intensity=m["intensity"]))
            continue
        d: dict[str, Any] = dict(id=nm, type="disney", color=list(m["base_color"]))
        for k in ("metallic", "roughness", "specular", "specular_tint", "sheen", "sheen_tint", "clearcoat",
                  "clearcoat_gloss", "spec_trans", "anisotropic", "diff_trans"):
            d[k] = float(m[k])
        d["ior"] = float(m["ior"])
        if m["transmission_color"] is not None:
            d["transmission_color"] = list(m["transmission_color"])
            d["transmission_depth"] = float(m["transmission_depth"])
        mats.append(d)
    ents = []
    for i, e in enumerate(world.entities):
        mname = world.material_names[e["material"]]
        if world.materials[e["material"]]["is_light_proxy"]:
            continue   # recreated by the area light
        if e["kind"] == ENT_QUAD:
            ents.append(dict(name=e["name"] or f"e{i}", type="quad", q=list(e["q"]), u=list(e["u"]),
                             v=list(e["v"]), material=mname))
        elif e["kind"] == ENT_SPHERE:
            ents.append(dict(name=e["name"] or f"e{i}", type="sphere", center=list(e["center"]),
                             radius=e["radius"], material=mname))
        else:
            from . import objfile
            fn = f"{name}_{i}.obj"
            sl = slice(e["first"], e["first"] + e["count"])
            nn = uv = None
            if world.tri_normals is not None:
                smooth = np.any(world.tri_normals[sl] != 0.0, axis=1)
                if smooth.any() and not smooth.all():
                    raise ValueError(f"mesh entity {i} mixes flat and smooth triangles, which one OBJ cannot "
                                     "express (ObjLoader drops a partial normal channel)")
                if smooth.all():
                    nn, uv = world.tri_normals[sl], world.tri_uvs[sl]
            objfile.write_obj(os.path.join(out_dir, fn), world.tri_verts[sl], nn, uv)
            ents.append(dict(name=e["name"] or f"e{i}", type="mesh", path=fn, material=mname))
    lights = []
    for l in world.lights:
        if l["type"] == LIGHT_AREA:
            lights.append(dict(type="area", corner=list(l["corner"]), u=list(l["u"]), v=list(l["v"]),
                               color=list(l["color"]), intensity=l["intensity"],
                               shadow_samples=l["shadow_samples"]))
        elif l["type"] == LIGHT_SPHERE:
            lights.append(dict(type="sphere", position=list(l["center"]), radius=l["radius"],
                               color=list(l["color"]), intensity=l["intensity"],
                               shadow_samples=l["shadow_samples"]))
        else:
            lights.append(dict(type="directional", direction=list(l["direction"]), color=list(l["color"]),
                               intensity=l["intensity"]))
    c = world.camera
    doc = dict(world=dict(sky=dict(type="flat", color=[float(x) for x in world.sky])),
               camera=dict(position=list(c["look_from"]), look_at=list(c["look_at"]), vup=list(c["vup"]),
                           fov=c["vfov"], aperture=c["aperture"], focal_dist=c["focus_dist"]),
               materials=mats, entities=ents, lights=lights)
    if world.medium:
        doc["world"]["medium"] = dict(type="homogeneous", sigma_a=list(world.medium["sigma_a"]),
                                      sigma_s=list(world.medium["sigma_s"]), g=world.medium["g"])
    path = os.path.join(out_dir, f"{name}.yaml")
    with open(path, "w") as f:
        yaml.safe_dump(doc, f, sort_keys=False)
    return path
