"""The display transform: Renderer.ToneMapToDisplay with AcesToneMap
(Rendering/Renderer.cs:741-751, 893-907) — exposure gain 2^ev (:333), floor
at zero, the ACES filmic fit, clamp to [0, 1], gamma 1/2.2.

CPU: the oracle's restatement against hand-derived values and a float32 numpy
transcription of the same formula. GPU: `rt_tonemap`, through the C-ABI,
against the oracle on random HDR values including negatives, values far above
the white point and several exposures. The two sides call different powf
implementations (CUDA and glibc), so they agree to a few float32 ulps."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import rt

abi = rt.abi


def hdr_values(h=61, w=67, seed=5):
    rng = np.random.default_rng(seed)
    x = np.exp(rng.uniform(np.log(1e-6), np.log(1e6), (3, h, w))).astype(np.float32)
    x[rng.random(x.shape) < 0.1] *= -1.0          # negatives: floored at zero
    x[rng.random(x.shape) < 0.05] = 0.0
    x[0, 0, :5] = [0.0, 1e-30, 0.18, 1.0, 1e6]
    return x


def numpy_aces(hdr, ev):
    f = np.float32
    c = hdr.astype(f) * f(2.0) ** f(ev)
    c = np.maximum(c, f(0))
    a = c * (f(2.51) * c + f(0.03))
    b = c * (f(2.43) * c + f(0.59)) + f(0.14)
    m = np.clip(a / b, f(0), f(1))
    return np.power(m, f(1) / f(2.2)).transpose(1, 2, 0)


def test_oracle_tonemap_fixed_points(oracle):
    x = np.zeros((3, 1, 4), np.float32)
    x[:, 0, 0] = 0.0          # black stays black: a/b = 0
    x[:, 0, 1] = -5.0         # floored at zero
    x[:, 0, 2] = 1e6          # far above white: a/b -> 2.51/2.43 > 1, clamped
    x[:, 0, 3] = 0.18
    y = oracle.tonemap(x, 0.0)
    assert np.all(y[0, 0] == 0) and np.all(y[0, 1] == 0) and np.all(y[0, 2] == 1.0)
    m = (0.18 * (2.51 * 0.18 + 0.03)) / (0.18 * (2.43 * 0.18 + 0.59) + 0.14)
    np.testing.assert_allclose(y[0, 3], m ** (1 / 2.2), rtol=1e-6)
    # one stop of exposure is a factor of two before the curve
    np.testing.assert_array_equal(oracle.tonemap(x * 2, 0.0), oracle.tonemap(x, 1.0))


@pytest.mark.parametrize("ev", [0.0, -2.5, 1.5])
def test_oracle_tonemap_matches_float32_formula(oracle, ev):
    x = hdr_values()
    np.testing.assert_allclose(oracle.tonemap(x, ev), numpy_aces(x, ev), rtol=2e-6, atol=1e-7)


@pytest.mark.gpu
@pytest.mark.parametrize("ev", [0.0, -2.5, 1.5, 4.0])
def test_rt_tonemap_matches_oracle(oracle, lib, ev):
    x = hdr_values(seed=int(abs(ev) * 10) + 7)
    h, w = x.shape[1:]
    out = np.zeros((h, w, 3), np.float32)
    abi.check(lib.rt_tonemap(abi.ptr(x), w, h, ev, abi.ptr(out)), "rt_tonemap")
    ref = oracle.tonemap(x, ev)
    assert np.all((out >= 0) & (out <= 1))
    np.testing.assert_allclose(out, ref, rtol=2e-6, atol=1e-7)
    assert np.array_equal(out == 0, ref == 0) and np.array_equal(out == 1, ref == 1)


def test_rt_tonemap_rejects_bad_arguments(lib):
    """Refused before any device work (runs without a GPU)."""
    x = np.zeros((3, 2, 2), np.float32)
    out = np.zeros((2, 2, 3), np.float32)
    assert lib.rt_tonemap(abi.ptr(x), 0, 2, 0.0, abi.ptr(out)) == -1
    assert lib.rt_tonemap(None, 2, 2, 0.0, abi.ptr(out)) == -1
