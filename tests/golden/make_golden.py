"""Generates tests/golden/oracle_golden.npz from the oracle (the C++
restatement of 3d-ray's C# hot path): Sobol draws, closest hits of fixed rays
on the Cornell box, Disney BSDF results for fixed queries, a 16x16x64-spp
Cornell film and the Kulla-Conty tables.

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def golden_inputs():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import random_rays, rt
    rng = np.random.default_rng(20261203)
    n = 4096
    inp = {"sobol_idx": rng.integers(0, 1 << 16, n).astype(np.uint32),
           "sobol_dim": rng.integers(0, 64, n).astype(np.uint32),
           "sobol_seed": rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32),
           "rays": random_rays(((1, 1, 1), (554, 554, 554)), 2048, seed=99)}
    q = np.zeros(2048, rt.abi.BSDF_QUERY_DTYPE)
    q["material"] = rng.integers(0, 3, 2048)
    q["front_face"] = 1
    q["pixel_seed"] = rng.integers(0, 1 << 32, 2048, dtype=np.uint64).astype(np.uint32)
    q["sample_index"] = rng.integers(0, 64, 2048)
    q["dim"] = rng.integers(2, 30, 2048)
    nrm = rng.normal(size=(2048, 3)).astype(np.float32)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    t = np.cross(nrm, rng.normal(size=(2048, 3))).astype(np.float32)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    v = rng.normal(size=(2048, 3)).astype(np.float32)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    v[np.sum(v * nrm, 1) < 0] *= -1
    l = rng.normal(size=(2048, 3)).astype(np.float32)
    l /= np.linalg.norm(l, axis=1, keepdims=True)
    q["n"], q["tangent"], q["bitangent"], q["v"], q["l"] = nrm, t, np.cross(nrm, t), v, l
    inp["bsdf"] = q
    return inp


def main():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, ROOT)
    from conftest import rt
    from oracle import binding
    binding.build()
    inp = golden_inputs()
    world = rt.scenes.cornell()
    osc = binding.OracleScene(rt.abi.PackedWorld(world))
    hits, _ = osc.trace_closest(inp["rays"])
    bsdf = osc.bsdf(inp["bsdf"], rt.abi.BSDF_RESULT_DTYPE)
    img, _ = osc.render(rt.abi.render_params(16, 16, 64, 8), threads=4)
    e, ea = binding.energy_lut()
    np.savez_compressed(os.path.join(HERE, "oracle_golden.npz"),
                        sobol=binding.sobol(inp["sobol_idx"], inp["sobol_dim"], inp["sobol_seed"]),
                        hits=hits, bsdf=bsdf, image=img, lut_e=e, lut_eavg=ea)


if __name__ == "__main__":
    main()
