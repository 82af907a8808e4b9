"""GPU FFT, pulse compression and Hermite upsampling through the C ABI against the oracle."""
import numpy as np
import pytest

import bsar
from bsar import scene as S

pytestmark = pytest.mark.gpu

from conftest import rel_l2


@pytest.fixture(scope="module")
def sc():
    return S.make_scene(S.scaled(S.config_spec(1), n_pulses=24))


def test_spline_bitexact(ctx, oracle, sc):
    x = sc.raw[:8]
    assert np.array_equal(ctx.spline_upsample(x, 4), oracle.spline_upsample(x, 4))
    y = sc.raw[:3, :37]                       # odd length, factor 3
    assert np.array_equal(ctx.spline_upsample(y, 3), oracle.spline_upsample(y, 3))


def test_spline_rejects_short_pulse(ctx):
    with pytest.raises(bsar.BsarError):
        ctx.spline_upsample(np.ones((1, 1), complex), 4)


@pytest.mark.parametrize("n", [2, 8, 256, 4096, 8192])
def test_fft_matches_oracle(ctx, oracle, n):
    rng = np.random.default_rng(n)
    x = rng.normal(size=(3, n)) + 1j * rng.normal(size=(3, n))
    for inv in (False, True):
        g = ctx.fft(x, inverse=inv)
        o = np.stack([oracle.fft(r, inverse=inv) for r in x])
        assert rel_l2(g, o) < 1e-13


def test_fft_known_answers(ctx):
    n = 1024
    d = np.zeros((1, n), complex)
    d[0, 0] = 1.0
    assert np.allclose(ctx.fft(d), 1.0, atol=1e-15)            # delta -> flat spectrum
    k = 37
    tone = np.exp(2j * np.pi * k * np.arange(n) / n)[None, :]
    F = ctx.fft(tone)
    assert abs(F[0, k] - n) < 1e-9 and np.abs(np.delete(F[0], k)).max() < 1e-9


def test_fft_non_power_of_two_unchanged(ctx):
    x = np.arange(12, dtype=complex).reshape(1, 12)
    assert np.array_equal(ctx.fft(x), x)
    assert "power of 2" in ctx.last_error()


@pytest.mark.parametrize("conj", [True, False])
def test_fft_correlate_matches_oracle(ctx, oracle, sc, conj):
    g = ctx.fft_correlate(sc.raw[:6], sc.reference, conj=conj)
    o = oracle.fft_correlate(sc.raw[:6], sc.reference, conj=conj)
    assert rel_l2(g, o) < 1e-12
    # ragged: signal shorter than the reference, non-power-of-two lengths
    g = ctx.fft_correlate(sc.raw[:2, :1000], sc.reference[:1500], conj=conj)
    o = oracle.fft_correlate(sc.raw[:2, :1000], sc.reference[:1500], conj=conj)
    assert rel_l2(g, o) < 1e-12


def test_matched_filter_peak_at_lag_zero(ctx, sc):
    out = ctx.fft_correlate(sc.reference[None, :], sc.reference)
    assert int(np.argmax(np.abs(out[0]))) == 0


def test_scene_compress_upsample_matches_oracle(ctx, oracle, sc):
    sid = bsar.upload_scene(ctx, sc)
    try:
        ctx.scene_compress(sid, "fp64")
        up = ctx.scene_read_upsampled(sid, sc.spec.n_pulses, sc.spec.n_samples * 4)
    finally:
        ctx.scene_release(sid)
    o = oracle.spline_upsample(oracle.fft_correlate(sc.raw, sc.reference), 4)
    assert rel_l2(up, o) < 1e-12
