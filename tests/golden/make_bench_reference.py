"""Generates the oracle's renders of the frames that bench.py's time-to-relMSE
measurements use as references, so that a GPU test can hold the bench's own
65 536-sample reference images to the oracle's noise floor:

- tests/golden/oracle_bench_cornell.npz: the Cornell box, 256x256, depth 8;
- tests/golden/oracle_bench_icospheres.npz: the 256x256 window at the centre
  of the 1920x1080 icosphere-field frame (the throughput scene), depth 12.

The oracle (the C++ restatement of the reference's bounce loop) renders each
frame twice, 2048 samples each, from the Sobol indices [2^21, 2^21 + 2048)
and [2^21 + 2048, 2^21 + 4096): disjoint from the bench's reference renders
([2^20, 2^20 + 65536)) and from its timed renders ([0, 16384)). Their mean is
a 4096-sample oracle image; their difference measures its noise pixel by
pixel.

Run from the repository root, naming the frames to make (default: both; about
five minutes for the Cornell box and ten for the icosphere window on eight
host cores):
    python tests/golden/make_bench_reference.py [cornell] [icospheres]
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

HALF_SPP = 2048
ORACLE_OFFSET = 1 << 21   # first Sobol index of the oracle's samples
GPU_OFFSET = 1 << 20      # first Sobol index of the bench's reference render
GPU_SPP = 65536           # samples of the bench's reference render

# name -> (film width, height, window (x0, y0, w, h), max depth)
FRAMES = {
    "cornell": (256, 256, (0, 0, 256, 256), 8),
    "icospheres": (1920, 1080, ((1920 - 256) // 2, (1080 - 256) // 2, 256, 256), 12),
}

# kept for the Cornell frame's callers
WIDTH, HEIGHT, DEPTH = 256, 256, 8


def path(name):
    return os.path.join(HERE, f"oracle_bench_{name}.npz")


def world(name="cornell"):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import rt
    return rt.scenes.cornell() if name == "cornell" else rt.scenes.throughput_scene()


def window_params(abi, name, spp, offset, **kw):
    """Render parameters of frame `name`: its film and window."""
    W, H, (x0, y0, ww, wh), depth = FRAMES[name]
    win = {} if (ww, wh) == (W, H) else dict(pixel_x0=x0, pixel_y0=y0, window_w=ww, window_h=wh)
    return abi.render_params(W, H, spp, depth, spp_offset=offset, **win, **kw)


def main(names):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import rt
    from oracle import binding
    binding.build()
    for name in names:
        W, H, (x0, y0, ww, wh), depth = FRAMES[name]
        osc = binding.OracleScene(rt.abi.PackedWorld(world(name)))
        halves = []
        for k in range(2):
            t0 = time.time()
            img, _ = osc.render(window_params(rt.abi, name, HALF_SPP, ORACLE_OFFSET + k * HALF_SPP))
            halves.append(np.asarray(img, np.float32)[:, y0:y0 + wh, x0:x0 + ww].copy())
            print(f"{name} half {k}: {time.time() - t0:.1f} s, mean {np.mean(halves[-1]):.5f}", flush=True)
        osc.close()
        np.savez_compressed(path(name), width=W, height=H, window=np.array([x0, y0, ww, wh]), depth=depth,
                            half_spp=HALF_SPP, oracle_offset=ORACLE_OFFSET, gpu_offset=GPU_OFFSET, gpu_spp=GPU_SPP,
                            a=halves[0], b=halves[1])


if __name__ == "__main__":
    main(sys.argv[1:] or list(FRAMES))
