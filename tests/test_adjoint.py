"""The path-replay adjoint (rt_adjoint) through the C-ABI.

- The parameter vector: get/set round trips exactly, and a scene changed with
  rt_scene_set_params renders exactly like one created from the changed world.
- Gradients of a linear image loss against central finite differences under
  common random numbers (same Sobol samples at theta +- eps), both on the GPU
  forward and on the CPU oracle.
- The torch.autograd.Function of the gradient-check harness.

Renders use the megakernel, whose per-pixel sums run in a fixed order, so the
finite differences carry no summation noise.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rt

pytestmark = pytest.mark.gpu
abi = rt.abi

SPHERE = dict(base_color=(0.6, 0.3, 0.2), roughness=0.4, metallic=0.2, specular=0.6, sheen=0.3)
NO_CLAMP = dict(max_sample_radiance=1e30, indirect_clamp_factor=1.0)


def _params(w, h, spp, depth=8, **kw):
    return abi.render_params(w, h, spp, depth, kernel=abi.KERNEL_MEGAKERNEL, **kw)


def _weights(h, w, seed=1):
    return np.random.default_rng(seed).uniform(0.0, 1.0, (3, h, w)).astype(np.float32)


def _fd(ds, rp, wimg, theta, i, eps):
    def loss(th):
        ds.set_params(th)
        return float((ds.render(rp).astype(np.float64) * wimg).sum())
    tp, tm = theta.copy(), theta.copy()
    tp[i] += eps
    tm[i] -= eps
    g = (loss(tp) - loss(tm)) / (2.0 * eps)
    ds.set_params(theta)
    return g


# --- the parameter vector -------------------------------------------------------
@pytest.mark.parametrize("scene", ["sphere", "volume"])
def test_param_vector_round_trip_is_exact(scene):
    w = rt.scenes.cornell_sphere(SPHERE) if scene == "sphere" else rt.scenes.cornell_volume()
    ds = rt.DiffScene(w)
    rp = _params(48, 48, 8)
    theta = ds.get_params()
    img0 = ds.render(rp)
    ds.set_params(theta)
    assert np.array_equal(ds.get_params(), theta)
    assert np.array_equal(ds.render(rp), img0)
    if scene == "volume":
        assert ds.get_params()[ds.medium_slot("sigma_s", 1)] == np.float32(0.016)
        np.testing.assert_allclose(theta[ds.slot("glass", "absorption"):ds.slot("glass", "absorption") + 3],
                                   [0.1, 0.3, 0.5], rtol=1e-5)


def test_set_params_renders_like_a_fresh_scene():
    w = rt.scenes.cornell_sphere(SPHERE)
    ds = rt.DiffScene(w)
    theta = ds.get_params()
    new = theta.copy()
    new[ds.slot("fit_sphere", "base_color", 1)] = 0.45
    new[ds.slot("fit_sphere", "roughness")] = 0.7
    new[ds.slot("fit_sphere", "metallic")] = 0.6
    new[ds.slot("fit_sphere", "sheen")] = 0.1
    new[ds.slot("light", "radiance", 0)] = 19.0
    new[ds.slot("red", "specular")] = 0.9
    ds.set_params(new)
    rp = _params(64, 64, 16)
    got = ds.render(rp)
    fresh = rt.DiffScene(rt.adjoint.world_with_params(w, new, theta))
    assert np.array_equal(fresh.get_params(), new)
    assert np.array_equal(got, fresh.render(rp))


def test_bad_vectors_are_rejected():
    ds = rt.DiffScene(rt.scenes.cornell_sphere(SPHERE))
    short = np.zeros(3, np.float32)
    assert ds.lib.rt_scene_set_params(ds.handle, abi.ptr(short), 3) == -1   # RT_ERR_INVALID_ARG
    assert ds.lib.rt_scene_get_params(ds.handle, abi.ptr(short), 3) == -1
    theta = ds.get_params()
    bad = theta.copy()
    bad[0] = np.nan
    with pytest.raises(abi.RtError):
        ds.set_params(bad)
    assert np.array_equal(ds.get_params(), theta)


# --- gradients against finite differences ------------------------------------------
def test_radiance_gradient_is_exact_without_clamps():
    """With the luminance clamps off the image is linear in the emitted
    radiance, so central differences are exact and the adjoint must match
    them to float rounding."""
    ds = rt.DiffScene(rt.scenes.cornell_sphere(SPHERE))
    rp = _params(64, 64, 64, **NO_CLAMP)
    wimg = _weights(64, 64)
    theta = ds.get_params()
    slots = [ds.slot("light", "radiance", c) for c in range(3)]
    g = ds.adjoint(rp, wimg, slots)
    for i in slots:
        fd = _fd(ds, rp, wimg, theta, i, 1e-3 * theta[i])
        assert g[i] == pytest.approx(fd, rel=2e-3)


@pytest.mark.parametrize("scene", ["sphere", "volume", "sky", "many_materials"])
def test_wavefront_adjoint_equals_megakernel(scene):
    """The wavefront form (a recording forward pass, then the replay with the
    shadow rays inline) computes the same per-vertex gradient terms as the
    megakernel on the same samples; only the order of the float sums differs
    (and the primal's shadow terms, which occlude adds in any order)."""
    if scene == "sphere":
        ds = rt.DiffScene(rt.scenes.cornell_sphere(SPHERE))
        slots = [ds.slot("fit_sphere", n) for n in ("roughness", "metallic", "specular", "sheen")]
        slots += [ds.slot("fit_sphere", "base_color", c) for c in range(3)]
        slots += [ds.slot("light", "radiance", c) for c in range(3)]
        res, spp, depth, kw = 48, 64, 8, {}
    elif scene == "volume":
        ds = rt.DiffScene(rt.scenes.cornell_volume())
        slots = [ds.medium_slot(k, c) for k in ("sigma_a", "sigma_s") for c in range(3)]
        slots += [ds.slot("glass", "absorption", c) for c in range(3)]
        res, spp, depth, kw = 32, 64, 16, {}
    elif scene == "sky":
        ds = rt.DiffScene(rt.scenes.sky_scene())
        slots = [ds.slot("red", "base_color", 0), ds.slot("ground", "base_color", 1)]
        res, spp, depth, kw = 32, 64, 8, NO_CLAMP
    else:   # more slots than the per-thread accumulators hold: the shared-memory gather
        w = rt.scenes.cornell_spheres()
        for k in range(2):
            w.add_material(f"unused{k}", rt.scenes.disney((0.5, 0.5, 0.5)))
        ds = rt.DiffScene(w)
        slots = None
        res, spp, depth, kw = 32, 32, 8, {}
    if scene == "many_materials":
        assert ds.count > rt.adjoint.ADJ_LOCAL_SLOTS
    wimg = _weights(res, res)
    mega = ds.adjoint(_params(res, res, spp, depth, spp_offset=7, **kw), wimg, slots)
    wf_rp = abi.render_params(res, res, spp, depth, kernel=abi.KERNEL_WAVEFRONT, spp_offset=7, **kw)
    wave = ds.adjoint(wf_rp, wimg, slots)
    assert ds.last_stats.kernel_launches > 4   # the two wavefront passes ran
    assert np.count_nonzero(mega) > 0
    np.testing.assert_allclose(wave, mega, rtol=1e-3, atol=1e-5 * np.abs(mega).max())


def test_wavefront_adjoint_runs_in_chunks_of_whole_spp_slices():
    """A request larger than the wavefront adjoint's sample record (2^24
    samples) is done in runs of whole spp slices; the gradient is the mean over
    all samples, so it equals the mean of the two halves rendered as separate
    calls."""
    ds = rt.DiffScene(rt.scenes.cornell_sphere(SPHERE))
    slots = [ds.slot("fit_sphere", "base_color", c) for c in range(3)] + [ds.slot("fit_sphere", "roughness")]
    res, spp = 64, 8192   # 2^25 samples: two runs
    wimg = _weights(res, res)

    def grad(n, off):
        return ds.adjoint(abi.render_params(res, res, n, 8, kernel=abi.KERNEL_WAVEFRONT, spp_offset=off), wimg,
                          slots).astype(np.float64)
    whole = grad(spp, 0)
    halves = 0.5 * (grad(spp // 2, 0) + grad(spp // 2, spp // 2))
    np.testing.assert_allclose(whole[slots], halves[slots], rtol=1e-4)


def test_medium_albedo_gradient_is_exact_without_roulette():
    """The medium's albedo at a fixed sigma_t (DiffScene.medium_albedo_direction)
    moves no free-flight density, so without Russian roulette every sample's
    value is smooth in it and Richardson central differences on the same
    samples match the adjoint to float rounding."""
    ds = rt.DiffScene(rt.scenes.cornell_volume())
    res = 32
    kw = dict(rr_min_bounces=1000, **NO_CLAMP)
    rp = _params(res, res, 256, 16, **kw)
    rw = abi.render_params(res, res, 256, 16, kernel=abi.KERNEL_WAVEFRONT, **kw)
    wimg = _weights(res, res)
    theta = ds.get_params()
    for c in range(3):
        dirs = ds.medium_albedo_direction(theta, c)
        adj = ds.medium_albedo_gradient(theta, ds.adjoint(rp, wimg, list(dirs)), c)
        eps = 1e-2 * float(theta[ds.medium_slot("sigma_s", c)]) / dirs[ds.medium_slot("sigma_s", c)]

        def loss(h):
            th = theta.copy()
            for i, k in dirs.items():
                th[i] = np.float32(float(theta[i]) + h * k)
            ds.set_params(th)
            return float((ds.render(rw).astype(np.float64) * wimg).sum())
        d1 = (loss(eps) - loss(-eps)) / (2 * eps)
        d2 = (loss(2 * eps) - loss(-2 * eps)) / (4 * eps)
        ds.set_params(theta)
        fd = (4 * d1 - d2) / 3
        assert adj == pytest.approx(fd, rel=2e-3), (c, adj, fd)


def test_unmasked_slots_come_back_zero():
    ds = rt.DiffScene(rt.scenes.cornell_sphere(SPHERE))
    rp = _params(32, 32, 16)
    slots = [ds.slot("fit_sphere", "base_color", 0)]
    g = ds.adjoint(rp, _weights(32, 32), slots)
    assert g[slots[0]] != 0.0
    assert np.count_nonzero(g) == 1


def test_autograd_function_matches_adjoint():
    import torch
    ds = rt.DiffScene(rt.scenes.cornell_sphere(SPHERE))
    rp = _params(48, 48, 16)
    theta0 = ds.get_params()
    target = torch.from_numpy(ds.render(rp))
    theta = theta0.copy()
    theta[ds.slot("fit_sphere", "base_color", 0)] = 0.3
    slots = [ds.slot("fit_sphere", n) for n in ("base_color", "roughness", "metallic")]
    fn = rt.adjoint.render_function()
    t = torch.tensor(theta, requires_grad=True)
    img = fn.apply(t, ds, rp, slots)
    loss = ((img - target) ** 2).sum()
    loss.backward()
    want = ds.adjoint(rp, (2.0 * (img.detach() - target)).numpy(), slots)
    # two adjoint runs differ only in the order of their block-level float sums
    np.testing.assert_allclose(t.grad.numpy(), want, rtol=1e-4, atol=1e-6 * np.abs(want).max())
    assert t.grad[slots[0]] < 0.0   # red was lowered: raising it lowers the loss


def _batches(ds, rp, wimg, theta, slots, eps_of, k, spp0=1 << 20):
    """Adjoint and central-difference gradients on k independent Sobol sample
    batches (spp_offset apart): arrays [k, len(slots)]."""
    adj, fd = [], []
    for b in range(k):
        rp.spp_offset = spp0 + b * rp.spp
        g = ds.adjoint(rp, wimg, slots)
        adj.append([g[i] for i in slots])
        fd.append([_fd(ds, rp, wimg, theta, i, eps_of(i)) for i in slots])
    return np.array(adj, np.float64), np.array(fd, np.float64)


def _agree(adj, fd, rel_floor):
    """The adjoint and the finite differences estimate the same gradient: the
    mean per-batch difference is within 4 standard errors (plus a relative
    floor for the finite differences' own truncation and rounding)."""
    d = adj - fd
    k = d.shape[0]
    se = d.std(axis=0, ddof=1) / np.sqrt(k)
    return np.abs(d.mean(axis=0)) <= 4.0 * se + rel_floor * np.abs(fd.mean(axis=0))


def test_sphere_bsdf_gradients_match_finite_differences():
    """C4's sphere parameters. baseColor does not change the sampling
    distributions, so eps = 1e-3 differences are tight; the lobe-weight
    parameters move the lobe choice, whose jumps make eps = 1e-3 differences
    noisy, so they use eps = 1e-2."""
    ds = rt.DiffScene(rt.scenes.cornell_sphere(SPHERE))
    rp = _params(64, 64, 256)
    wimg = _weights(64, 64)
    theta = ds.get_params()
    base = [ds.slot("fit_sphere", "base_color", c) for c in range(3)]
    lobes = [ds.slot("fit_sphere", n) for n in ("roughness", "metallic", "specular", "sheen")]
    adj, fd = _batches(ds, rp, wimg, theta, base + lobes, lambda i: 1e-3 if i in base else 1e-2, 6)
    ok = _agree(adj, fd, 5e-3)
    assert ok.all(), (adj.mean(0), fd.mean(0))
    # baseColor moves no sampling distribution except Russian roulette: each
    # batch of 1 M samples alone is within 3e-2
    np.testing.assert_allclose(adj[:, :3], fd[:, :3], rtol=3e-2)


def test_volume_gradients_match_finite_differences():
    """C5: the medium's sigma_a and sigma_s and the glass sphere's
    absorption, with the clamps off."""
    ds = rt.DiffScene(rt.scenes.cornell_volume())
    rp = _params(48, 48, 512, **NO_CLAMP)
    wimg = np.ones((3, 48, 48), np.float32)
    theta = ds.get_params()
    slots = [ds.medium_slot("sigma_a", 0), ds.medium_slot("sigma_s", 0), ds.slot("glass", "absorption", 0)]
    adj, fd = _batches(ds, rp, wimg, theta, slots, lambda i: 1e-2 * theta[i], 6)
    assert _agree(adj, fd, 5e-3).all(), (adj.mean(0), fd.mean(0))
    assert adj.mean(0)[0] < 0 and adj.mean(0)[2] <= 0   # more absorption darkens the box


def test_gradients_match_cpu_oracle_finite_differences(oracle):
    """Central differences of the CPU oracle (the reference's loop restated)
    on the same samples: emitter radiance without clamps (exact) and the
    sphere's baseColor with the reference's clamps."""
    w = rt.scenes.cornell_sphere(SPHERE)
    ds = rt.DiffScene(w)
    theta = ds.get_params()
    wimg = _weights(24, 24, seed=3)

    def cpu_grad(rp, i, eps):
        vals = []
        for sgn in (1.0, -1.0):
            th = theta.copy()
            th[i] += sgn * eps
            osc = oracle.OracleScene(abi.PackedWorld(rt.adjoint.world_with_params(w, th, theta)))
            img, _ = osc.render(rp)
            osc.close()
            vals.append(float((np.asarray(img, np.float64).reshape(3, 24, 24) * wimg).sum()))
        return (vals[0] - vals[1]) / (2.0 * eps)

    rp = _params(24, 24, 256, **NO_CLAMP)
    i = ds.slot("light", "radiance", 1)
    g = ds.adjoint(rp, wimg, [i])[i]
    assert g == pytest.approx(cpu_grad(rp, i, 1e-3 * theta[i]), rel=2e-3)
    rp = _params(24, 24, 1024)
    i = ds.slot("fit_sphere", "base_color", 0)
    g = ds.adjoint(rp, wimg, [i])[i]
    assert g == pytest.approx(cpu_grad(rp, i, 1e-3), rel=2e-2)


def test_emissive_sphere_radiance_gradient_is_exact():
    """An emissive sphere (cone-sampled geometry light): its radiance enters
    through NEE and through BSDF rays that hit it; without the clamps the
    image is linear in it."""
    w = rt.scenes.cornell_sphere(SPHERE)
    glow = w.add_material("glow", rt.scenes.emissive((6.0, 4.0, 2.0), 1.0))
    w.add_sphere((150, 420, 300), 40.0, glow, name="glow")
    ds = rt.DiffScene(w)
    rp = _params(48, 48, 64, **NO_CLAMP)
    wimg = _weights(48, 48, seed=5)
    theta = ds.get_params()
    slots = [ds.slot("glow", "radiance", c) for c in range(3)]
    g = ds.adjoint(rp, wimg, slots)
    for i in slots:
        assert g[i] == pytest.approx(_fd(ds, rp, wimg, theta, i, 1e-3 * theta[i]), rel=2e-3)


def test_gradients_under_a_flat_sky_match_finite_differences():
    """The flat sky adds a term at every miss; the replay's suffix must carry
    it into the factor gradients of the surfaces before the miss."""
    w = rt.scenes.sky_scene()
    ds = rt.DiffScene(w)
    rp = _params(48, 32, 256, **NO_CLAMP)
    wimg = np.ones((3, 32, 48), np.float32)
    theta = ds.get_params()
    slots = [ds.slot("red", "base_color", 0), ds.slot("ground", "base_color", 1)]
    adj, fd = _batches(ds, rp, wimg, theta, slots, lambda i: 1e-3, 6)
    assert _agree(adj, fd, 5e-3).all(), (adj.mean(0), fd.mean(0))
    assert (adj.mean(0) > 0).all()   # brighter albedo, brighter image


def _sign_weights(ds, theta, i, eps, res, depth, **kw):
    """A loss weighting for parameter i: the sign of its central-difference
    image from an independent GPU pilot render, so that every pixel's change
    adds to dL/dtheta instead of partly cancelling (a fixed weighting: the
    pilot's Sobol range is disjoint from the checks')."""
    pilot = abi.render_params(res, res, 4096, depth, kernel=abi.KERNEL_WAVEFRONT, spp_offset=1 << 24, **kw)
    films = []
    for sgn in (1.0, -1.0):
        th = theta.copy()
        th[i] += sgn * eps
        ds.set_params(th)
        films.append(ds.render(pilot).astype(np.float64))
    ds.set_params(theta)
    return np.sign(films[0] - films[1]).astype(np.float32)


def _oracle_fd(oracle, world, theta, i, eps, rp, wimg):
    vals = []
    for sgn in (1.0, -1.0):
        th = theta.copy()
        th[i] += sgn * eps
        osc = oracle.OracleScene(abi.PackedWorld(rt.adjoint.world_with_params(world, th, theta)))
        img, _ = osc.render(rp)
        osc.close()
        vals.append(float((np.asarray(img, np.float64) * wimg).sum()))
    return (vals[0] - vals[1]) / (2.0 * eps)


@pytest.mark.parametrize("name", ["roughness", "metallic", "specular", "sheen"])
def test_lobe_parameter_gradients_match_cpu_oracle_finite_differences(oracle, name):
    """The sphere's lobe-weight parameters (they move the lobe choice, so the
    differences carry the jumps of lobes that flip): the GPU adjoint against
    central differences of the CPU oracle on the same Sobol samples, in 6
    batches, within 4 standard errors of their per-batch difference plus 2e-2
    of the truncation that eps = 2e-2 leaves."""
    w = rt.scenes.cornell_sphere(SPHERE)
    ds = rt.DiffScene(w)
    theta = ds.get_params()
    i = ds.slot("fit_sphere", name)
    eps, res = 2e-2, 24
    wimg = _sign_weights(ds, theta, i, eps, res, 8)
    adj, fd = [], []
    for b in range(6):
        rp = _params(res, res, 1024, spp_offset=(1 << 20) + b * 1024)
        adj.append(ds.adjoint(rp, wimg, [i])[i])
        fd.append(_oracle_fd(oracle, w, theta, i, eps, rp, wimg))
    adj, fd = np.array(adj)[:, None], np.array(fd)[:, None]
    assert _agree(adj, fd, 2e-2).all(), (name, adj.ravel(), fd.ravel())
    assert abs(fd.mean()) > 0.0


def test_medium_gradient_matches_cpu_oracle_finite_differences(oracle):
    """C5's medium scattering coefficient (red), clamps off: the GPU adjoint
    against central differences of the CPU oracle on the same samples."""
    w = rt.scenes.cornell_volume()
    ds = rt.DiffScene(w)
    theta = ds.get_params()
    i = ds.medium_slot("sigma_s", 0)
    eps, res = 1e-2 * float(theta[i]), 24
    wimg = _sign_weights(ds, theta, i, eps, res, 16, **NO_CLAMP)
    adj, fd = [], []
    for b in range(6):
        rp = _params(res, res, 512, depth=16, spp_offset=(1 << 20) + b * 512, **NO_CLAMP)
        adj.append(ds.adjoint(rp, wimg, [i])[i])
        fd.append(_oracle_fd(oracle, w, theta, i, eps, rp, wimg))
    adj, fd = np.array(adj)[:, None], np.array(fd)[:, None]
    assert _agree(adj, fd, 2e-2).all(), (adj.ravel(), fd.ravel())
