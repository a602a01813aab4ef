"""The C-ABI surface: the library loads without a GPU, exports every symbol
include/rt3d.h declares, the ctypes mirror matches the header's layouts, and
calls that need a device fail cleanly (no trap) when there is none."""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu, rt

abi = rt.abi


def declared_functions():
    src = open(os.path.join(ROOT, "include", "rt3d.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rt_[a-z_0-9]+)\s*\(", src)))


def test_all_declared_symbols_exported(lib):
    names = declared_functions()
    assert len(names) >= 18
    for n in names:
        assert hasattr(lib, n), n


def test_abi_version(lib):
    assert lib.rt_abi_version() == 2


@pytest.mark.parametrize("struct,size", [("RtMaterialDesc", 120), ("RtEntityDesc", 80), ("RtLightDesc", 104),
                                         ("RtCameraDesc", 48), ("RtMediumDesc", 36), ("RtRenderParams", 112),
                                         ("RtStats", 144), ("RtBsdfQuery", 96), ("RtBsdfResult", 80),
                                         ("RtRequest", 72), ("RtSceneInfo", 64), ("RtWorldDesc", 184),
                                         ("RtCapture", 64), ("RtSceneOptions", 32), ("RtMediumQuery", 40),
                                         ("RtMediumResult", 56)])
def test_struct_sizes(struct, size):
    """Sizes of the C structs (checked against the header by the C compiler in
    the build: see the static_asserts in kernels.cu)."""
    assert C.sizeof(getattr(abi, struct)) == size


def test_no_device_fails_cleanly(lib):
    if has_gpu():
        pytest.skip("a device is present")
    h = C.c_void_p()
    rc = lib.rt_scene_create(abi.PackedWorld(rt.scenes.cornell()).ref(), C.byref(h))
    assert rc == -8 and h.value is None
    assert b"device" in lib.rt_last_error()


def test_renderer_params_mirror_reference_defaults():
    p = rt.abi.render_params(8, 8, 4, 3)
    assert p.max_sample_radiance == 10.0 and abs(p.indirect_clamp_factor - 0.25) < 1e-7
    assert p.rr_min_bounces == -1 and p.sort_materials == -1
    assert p.iteration_limit == 0 and p.shadow_queue_limit == 0   # the test-only limits are off
