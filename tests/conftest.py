"""Test setup: loads the package (directory 3d-ray_b200/, module rt3d_b200),
registers the `gpu` marker and provides shared scene fixtures.

CPU tests (-m "not gpu") check the oracle against the reference's own test
properties, the host-side world assembly against the oracle, and the C-ABI
surface. GPU tests (-m gpu) call the CUDA path through the C-ABI and compare
it with the oracle on the same inputs.
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def load_package():
    if "rt3d_b200" in sys.modules:
        return sys.modules["rt3d_b200"]
    pkg_dir = os.path.join(ROOT, "3d-ray_b200")
    spec = importlib.util.spec_from_file_location("rt3d_b200", os.path.join(pkg_dir, "__init__.py"),
                                                  submodule_search_locations=[pkg_dir])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["rt3d_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


rt = load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def pkg():
    return rt


@pytest.fixture(scope="session")
def oracle():
    from oracle import binding
    binding.build()
    return binding


@pytest.fixture(scope="session")
def lib():
    return rt.abi.load()


@pytest.fixture(scope="session")
def cornell_world():
    return rt.scenes.cornell()


@pytest.fixture(scope="session")
def throughput_world_small():
    """C2 construction at reduced size (8 spheres, level 3) for fast tests."""
    return rt.scenes.throughput_scene(n_spheres=8, level=3)


@pytest.fixture(scope="session")
def throughput_world():
    return rt.scenes.throughput_scene()


def camera_rays(world, width, height, seed=1, jitter=True):
    """Camera rays of the reference pinhole camera (Camera.cs:127-139) in
    float32 numpy arithmetic: 8 floats per ray (o, d, pad)."""
    c = world.camera
    f32 = np.float32
    from_ = np.array(c["look_from"], f32)
    at = np.array(c["look_at"], f32)
    vup = np.array(c["vup"], f32)
    theta = f32(c["vfov"]) * f32(np.pi) / f32(180)
    h = np.tan(theta / f32(2), dtype=f32)
    vh = f32(2) * h
    vw = f32(width / height) * vh
    w = from_ - at
    w = w / np.sqrt(np.sum(w * w, dtype=f32), dtype=f32)
    u = np.cross(vup, w).astype(f32)
    u = u / np.sqrt(np.sum(u * u, dtype=f32), dtype=f32)
    v = np.cross(w, u).astype(f32)
    fd = f32(c["focus_dist"])
    hor = fd * vw * u
    ver = fd * vh * v
    llc = from_ - hor / f32(2) - ver / f32(2) - fd * w
    rng = np.random.default_rng(seed)
    ii, jj = np.meshgrid(np.arange(width), np.arange(height))
    ju = rng.random(ii.shape, dtype=np.float32) if jitter else np.full(ii.shape, 0.5, f32)
    jv = rng.random(ii.shape, dtype=np.float32) if jitter else np.full(ii.shape, 0.5, f32)
    s = (ii.astype(f32) + ju) / f32(width)
    t = ((height - jj - 1).astype(f32) + jv) / f32(height)
    tgt = llc + s[..., None] * hor + t[..., None] * ver
    d = tgt - from_
    rays = np.zeros((width * height, 8), f32)
    rays[:, 0:3] = from_
    rays[:, 3:6] = d.reshape(-1, 3)
    return rays


def random_rays(world_box, n, seed=2):
    """Rays from random points inside the scene box in random directions."""
    lo, hi = world_box
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True).astype(np.float32)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3:6] = d
    return rays
