"""Generates tests/golden/oracle_images.npz: high-sample oracle renders that the
image-parity test compares the GPU's 65 536-sample renders against.

For each scene below, the oracle (the C++ restatement of the reference's
bounce loop) renders the same frame twice, 2048 samples each, from the Sobol
indices [65536, 67584) and [67584, 69632): disjoint from the GPU's [0, 65536),
so the two estimates are independent. Their mean is a 4096-sample oracle image;
their difference measures its noise pixel by pixel.

Run from the repository root (takes a few minutes on all host cores):
    python tests/golden/make_reference_images.py
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

WIDTH = HEIGHT = 64
HALF_SPP = 2048
ORACLE_OFFSET = 65536     # first Sobol index of the oracle's samples
GPU_SPP = 65536           # the GPU renders Sobol indices [0, GPU_SPP)


def scenes():
    """name -> (world, max depth): C1, the C4 sphere box (sheen on), the flat
    sky with glass, spherical emitters, C5's medium and glass at the
    configured density and at a tenth of it."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import rt
    S = rt.scenes
    return {
        "cornell": (S.cornell(), 8),
        "cornell_sphere": (S.cornell_sphere(dict(base_color=(0.7, 0.4, 0.2), roughness=0.35, metallic=0.3,
                                                 specular=0.6, sheen=0.8)), 8),
        "sky": (S.sky_scene(), 8),
        "cornell_spheres": (S.cornell_spheres(), 8),
        "volume": (S.cornell_volume(), 16),
        "volume_thin": (S.cornell_volume(density=0.1), 16),
    }


def main():
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import rt
    from oracle import binding
    binding.build()
    out = {}
    for name, (world, depth) in scenes().items():
        t0 = time.time()
        osc = binding.OracleScene(rt.abi.PackedWorld(world))
        halves = []
        for k in range(2):
            p = rt.abi.render_params(WIDTH, HEIGHT, HALF_SPP, depth, spp_offset=ORACLE_OFFSET + k * HALF_SPP)
            img, _ = osc.render(p)
            halves.append(img)
        out[f"{name}_a"], out[f"{name}_b"] = halves
        print(f"{name}: {time.time() - t0:.1f} s, mean {np.mean(halves[0]):.4f} {np.mean(halves[1]):.4f}",
              flush=True)
    np.savez_compressed(os.path.join(HERE, "oracle_images.npz"), width=WIDTH, height=HEIGHT, half_spp=HALF_SPP,
                        oracle_offset=ORACLE_OFFSET, **out)


if __name__ == "__main__":
    main()
