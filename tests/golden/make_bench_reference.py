"""Generates tests/golden/oracle_bench_cornell.npz: the oracle's render of the
frame that bench.py's time-to-relMSE measurement uses as its reference (the
Cornell box, 256x256, depth 8), so that a GPU test can hold the bench's own
65 536-sample reference image to the oracle's noise floor.

The oracle (the C++ restatement of the reference's bounce loop) renders the
frame twice, 2048 samples each, from the Sobol indices [2^21, 2^21 + 2048)
and [2^21 + 2048, 2^21 + 4096): disjoint from the bench's reference render
([2^20, 2^20 + 65536)) and from its timed renders ([0, 256)). Their mean is a
4096-sample oracle image; their difference measures its noise pixel by pixel.

Run from the repository root (about five minutes on eight host cores):
    python tests/golden/make_bench_reference.py
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

WIDTH = HEIGHT = 256
DEPTH = 8
HALF_SPP = 2048
ORACLE_OFFSET = 1 << 21   # first Sobol index of the oracle's samples
GPU_OFFSET = 1 << 20      # first Sobol index of the bench's reference render
GPU_SPP = 65536           # samples of the bench's reference render


def world():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import rt
    return rt.scenes.cornell()


def main():
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import rt
    from oracle import binding
    binding.build()
    osc = binding.OracleScene(rt.abi.PackedWorld(world()))
    halves = []
    for k in range(2):
        t0 = time.time()
        p = rt.abi.render_params(WIDTH, HEIGHT, HALF_SPP, DEPTH, spp_offset=ORACLE_OFFSET + k * HALF_SPP)
        img, _ = osc.render(p)
        halves.append(np.asarray(img, np.float32))
        print(f"half {k}: {time.time() - t0:.1f} s, mean {np.mean(halves[-1]):.5f}", flush=True)
    osc.close()
    np.savez_compressed(os.path.join(HERE, "oracle_bench_cornell.npz"), width=WIDTH, height=HEIGHT, depth=DEPTH,
                        half_spp=HALF_SPP, oracle_offset=ORACLE_OFFSET, gpu_offset=GPU_OFFSET, gpu_spp=GPU_SPP,
                        a=halves[0], b=halves[1])


if __name__ == "__main__":
    main()
