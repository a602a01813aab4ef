"""Per-query parity of every Disney lobe and of the medium, through the C-ABI.

The BSDF half runs `rt_bsdf_batch` on the materials of `lobes.lobe_world()`:
sheen (the C4 sphere), smooth and rough specular transmission entered from
both sides (the C5 glass, total internal reflection from inside), a thin
sheet, diffuse transmission, anisotropic rotated GGX, clearcoat on both coat
paths, a rough metal's multiscatter, and one material with every lobe
(DisneyBsdf.cs:418-997, 1176-1709; Microfacet.cs:22-125; SheenCharlie.cs).
The north-star bar: the chosen lobe, IsDelta, the Transition and the Sobol
dimensions consumed equal the oracle's bit for bit; Evaluate, Pdf and
EvaluateDirect agree within 1e-4 relative.

The medium half runs `rt_medium_batch` on five media: HomogeneousMedium.Sample
and Transmittance (HomogeneousMedium.cs:36-76) and HenyeyGreensteinPhase.Sample
and Evaluate (HenyeyGreensteinPhase.cs:23-54) on identical Sobol streams; the
scatter decision and dimensions are exact, t and beta within 1e-5 relative,
the phase pdf and direction within 1e-4.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import lobes
from conftest import rt

abi = rt.abi

# Sampled directions go through cos/sin, where CUDA and glibc differ by ulps:
# a sampled direction agrees to ~1e-6, and the lobe values are compared at the
# GPU's own direction (the oracle evaluates it) within the BSDF tolerance.
RTOL = 1e-4
ATOL = 1e-7


def test_lobe_world_reaches_every_lobe_in_the_oracle(oracle):
    """The query set is strong enough: in the oracle, every lobe id 0..6 is
    sampled at least 1000 times, both transitions occur, and deltas and
    non-deltas are both common (CPU check of the GPU test's inputs)."""
    w = lobes.lobe_world()
    q = lobes.bsdf_queries(w, 200000)
    o = oracle.OracleScene(abi.PackedWorld(w)).bsdf(q, abi.BSDF_RESULT_DTYPE)
    counts = np.bincount(o["lobe"][o["lobe"] >= 0], minlength=7)
    assert np.all(counts >= 1000), dict(zip(lobes.LOBES, counts))
    tr = np.bincount(o["transition"], minlength=3)
    assert tr[1] > 1000 and tr[2] > 1000
    assert 0.1 < o["is_delta"].mean() < 0.9


def test_medium_oracle_batch_matches_free_functions(oracle):
    """The oracle's batch form draws exactly what its free functions give for
    the same uniforms (channel, distance; then the two phase draws)."""
    w = lobes.medium_world("chromatic_vacuum_channel")
    q = lobes.medium_queries(2000)
    o = oracle.OracleScene(abi.PackedWorld(w)).medium(q, abi.MEDIUM_RESULT_DTYPE)
    m = w.medium
    for i in range(0, 2000, 37):
        d = int(q["dim"][i])
        u = oracle.sobol(np.full(4, q["sample_index"][i]), np.arange(d, d + 4), q["pixel_seed"][i])
        ch = min(int(u[0] * np.float32(3)), 2)
        takes_distance = (m["sigma_a"][ch] + m["sigma_s"][ch]) > 0
        sc, t, beta = oracle.medium_sample(m["sigma_a"], m["sigma_s"], float(q["tmax"][i]), float(u[0]), float(u[1]))
        assert bool(o["scattered"][i]) == sc and o["t"][i] == np.float32(t)
        np.testing.assert_array_equal(o["beta"][i], beta)
        k = 2 if takes_distance else 1
        assert o["dims_used"][i] == k + 2
        wi, pdf = oracle.hg_sample(m["g"], q["wo"][i], float(u[k]), float(u[k + 1]))
        np.testing.assert_array_equal(o["phase_wi"][i], wi)
        assert o["phase_pdf"][i] == np.float32(pdf)
        assert o["phase_eval"][i] == np.float32(oracle.hg_eval(m["g"], q["wo"][i], q["wi"][i]))


class _Scene:
    def __init__(self, world):
        self.lib = abi.load()
        self.packed = abi.PackedWorld(world)
        h = C.c_void_p()
        abi.check(self.lib.rt_scene_create(self.packed.ref(), C.byref(h)), "rt_scene_create")
        self.h = h

    def close(self):
        self.lib.rt_scene_destroy(self.h)


@pytest.mark.gpu
def test_every_disney_lobe_matches_oracle(oracle):
    w = lobes.lobe_world()
    q = lobes.bsdf_queries(w, 200000)
    s = _Scene(w)
    try:
        g = np.zeros(q.shape[0], abi.BSDF_RESULT_DTYPE)
        abi.check(s.lib.rt_bsdf_batch(s.h, abi.ptr(q), q.shape[0], abi.ptr(g)), "rt_bsdf_batch")
    finally:
        s.close()
    osc = oracle.OracleScene(abi.PackedWorld(w))
    o = osc.bsdf(q, abi.BSDF_RESULT_DTYPE)
    counts = np.bincount(g["lobe"][g["lobe"] >= 0], minlength=7)
    assert np.all(counts >= 1000), dict(zip(lobes.LOBES, counts))
    for k in ("lobe", "has_sample", "is_delta", "dims_used", "transition"):
        bad = np.flatnonzero(g[k] != o[k])
        assert bad.size == 0, (k, bad[:10], q["material"][bad[:10]])
    for k in ("f", "pdf", "fd"):
        np.testing.assert_allclose(g[k], o[k], rtol=RTOL, atol=ATOL, err_msg=k)
    hs = g["has_sample"] == 1
    np.testing.assert_allclose(g["wo"][hs], o["wo"][hs], rtol=1e-4, atol=1e-5)
    # non-delta samples: the sample's f and pdf are Evaluate and Pdf at the
    # sampled direction; evaluate the oracle at the GPU's direction
    nd = hs & (g["is_delta"] == 0)
    q2 = q[nd].copy()
    q2["l"] = g["wo"][nd]
    o2 = osc.bsdf(q2, abi.BSDF_RESULT_DTYPE)
    np.testing.assert_allclose(g["s_pdf"][nd], o2["pdf"], rtol=RTOL, atol=ATOL)
    np.testing.assert_allclose(g["s_f"][nd], o2["f"], rtol=RTOL, atol=ATOL)
    # delta samples: the lobe's weight (Fresnel, tint, G1 of the sampled
    # direction, divided by the lobe probability floor). A rough transmission
    # weight holds G1 at the sampled direction, which the two sides draw a few
    # ulps apart; near grazing G1 turns that into more than 1e-4, so a few in
    # 1e5 weights there are held to 5e-2 instead.
    dl = hs & (g["is_delta"] == 1)
    gs, os_ = g["s_f"][dl], o["s_f"][dl]
    close = np.isclose(gs, os_, rtol=RTOL, atol=1e-6)
    assert close.mean() > 1 - 1e-4, close.mean()
    np.testing.assert_allclose(gs, os_, rtol=5e-2, atol=1e-6)
    far = np.flatnonzero(~np.all(close, axis=1))
    cos_far = np.abs(np.sum(g["wo"][dl][far] * q["n"][dl][far], axis=1))
    assert np.all(np.isin(q["material"][dl][far], [lobes.index("glass_rough"), lobes.index("glass_rough_aniso"),
                                                   lobes.index("thin_sheet"), lobes.index("everything")])), far
    assert far.size == 0 or np.max(cos_far) < 0.2, cos_far
    assert np.all(g["s_pdf"][dl] == 1.0)
    # per lobe, the sampled weights are not trivially zero
    for lobe in range(7):
        sel = hs & (g["lobe"] == lobe)
        assert np.count_nonzero(np.any(g["s_f"][sel] > 0, axis=1)) > 0.5 * sel.sum(), lobes.LOBES[lobe]


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(lobes.MEDIA))
def test_medium_and_phase_match_oracle(oracle, name):
    w = lobes.medium_world(name)
    q = lobes.medium_queries(100000)
    s = _Scene(w)
    try:
        g = np.zeros(q.shape[0], abi.MEDIUM_RESULT_DTYPE)
        abi.check(s.lib.rt_medium_batch(s.h, abi.ptr(q), q.shape[0], abi.ptr(g)), "rt_medium_batch")
    finally:
        s.close()
    o = oracle.OracleScene(abi.PackedWorld(w)).medium(q, abi.MEDIUM_RESULT_DTYPE)
    # a sampled distance within a few ulps of tmax may fall on either side
    # (logf differs by ulps between CUDA and glibc): a scatter decision may
    # differ only where the side that scattered drew a distance that close
    flip = g["scattered"] != o["scattered"]
    t_sc = np.where(g["scattered"] == 1, g["t"], o["t"])
    assert flip.mean() < 1e-3
    assert np.all(np.abs(t_sc[flip] - q["tmax"][flip]) <= 1e-5 * q["tmax"][flip])
    ok = ~flip
    assert np.array_equal(g["dims_used"], o["dims_used"])
    sc = o["scattered"] == 1
    assert 0.01 < sc.mean() < 0.99 or name == "forward_peaked"
    np.testing.assert_allclose(g["t"][ok], o["t"][ok], rtol=1e-5)
    np.testing.assert_allclose(g["beta"][ok], o["beta"][ok], rtol=1e-5, atol=1e-30)
    np.testing.assert_allclose(g["tr"], o["tr"], rtol=1e-5, atol=1e-30)
    np.testing.assert_allclose(g["phase_eval"], o["phase_eval"], rtol=1e-4)
    np.testing.assert_allclose(g["phase_wi"], o["phase_wi"], rtol=1e-4, atol=1e-5)
    # the phase pdf at the GPU's own direction (a forward-peaked lobe turns a
    # 1e-7 change of the direction into ~1e-4 of its pdf)
    g_ = w.medium["g"]
    pdf_at_gpu = np.array([oracle.hg_eval(g_, q["wo"][i], g["phase_wi"][i]) for i in range(q.shape[0])], np.float32)
    np.testing.assert_allclose(g["phase_pdf"], pdf_at_gpu, rtol=1e-4)
    np.testing.assert_allclose(g["phase_pdf"], o["phase_pdf"], rtol=2e-3)


@pytest.mark.gpu
def test_medium_batch_needs_a_medium():
    s = _Scene(rt.scenes.cornell())
    try:
        q = lobes.medium_queries(4)
        g = np.zeros(4, abi.MEDIUM_RESULT_DTYPE)
        assert s.lib.rt_medium_batch(s.h, abi.ptr(q), 4, abi.ptr(g)) == -1
        assert b"medium" in s.lib.rt_last_error()
    finally:
        s.close()
