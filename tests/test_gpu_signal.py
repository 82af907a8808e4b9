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


# 16384..65536 (FP64) run on clusters of 2, 4 and 8 CTAs
@pytest.mark.parametrize("n", [2, 8, 256, 4096, 8192, 16384, 32768, 65536])
def test_fft_matches_oracle(ctx, oracle, n):
    rng = np.random.default_rng(n)
    x = rng.normal(size=(3, n)) + 1j * rng.normal(size=(3, n))
    for inv in (False, True):
        g = ctx.fft(x, inverse=inv)
        o = np.stack([oracle.fft(r, inverse=inv) for r in x])
        # the reference's twiddle recurrence drifts with length; the device uses a table
        assert rel_l2(g, o) < (1e-13 if n <= 8192 else 1e-12)
        npy = np.fft.ifft(x, axis=1) if inv else np.fft.fft(x, axis=1)
        assert rel_l2(g, npy) < 1e-13


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


@pytest.mark.parametrize("ns,nref", [(12000, 16384), (16384, 1201), (30000, 2000)])
def test_fft_correlate_cluster_lengths(ctx, oracle, ns, nref):
    """Correlations whose padded length needs a 2- or 4-CTA cluster (FP64)."""
    rng = np.random.default_rng(ns + nref)
    x = rng.normal(size=(3, ns)) + 1j * rng.normal(size=(3, ns))
    r = rng.normal(size=nref) + 1j * rng.normal(size=nref)
    g = ctx.fft_correlate(x, r)
    o = oracle.fft_correlate(x, r)
    assert rel_l2(g, o) < 1e-12


def test_scene_compress_long_pulses(ctx, oracle):
    """16384-sample pulses: FP64 on a 2-CTA cluster, FP32 on one CTA, FP16 storage."""
    spec = S.scaled(S.config_spec(2), n_pulses=6, n_samples=16384, n_scatterers=8)
    sc = S.make_scene(spec)
    o = oracle.spline_upsample(oracle.fft_correlate(sc.raw, sc.reference), 4)
    sid = bsar.upload_scene(ctx, sc)
    try:
        got = {}
        for prec in ("fp64", "mixed", "mixed_fp16"):
            got[prec] = ctx.scene_read_stored(sid, spec.n_pulses, spec.n_samples * 4, prec)
    finally:
        ctx.scene_release(sid)
    assert rel_l2(got["fp64"], o) < 1e-12
    assert rel_l2(got["mixed"], o) < 1e-5
    assert rel_l2(got["mixed_fp16"], o) < 2e-3


@pytest.mark.parametrize("ns,factor", [(4096, 4), (8192, 4), (4096, 2), (8192, 8)])
def test_scene_compress_fp32_register_transforms(ctx, oracle, ns, factor):
    """FP32 pulses of 4096 and 8192 samples (the register-resident transforms; x4 with the
    16-byte epilogue stores, other factors with one store per output) into complex64 and
    FP16 storage, against the FP64 oracle."""
    spec = S.scaled(S.config_spec(2), n_pulses=5, n_samples=ns, n_scatterers=8, upsample=factor)
    sc = S.make_scene(spec)
    o = oracle.spline_upsample(oracle.fft_correlate(sc.raw, sc.reference), factor)
    sid = bsar.upload_scene(ctx, sc)
    try:
        m32 = ctx.scene_read_stored(sid, spec.n_pulses, ns * factor, "mixed")
        m16 = ctx.scene_read_stored(sid, spec.n_pulses, ns * factor, "mixed_fp16")
    finally:
        ctx.scene_release(sid)
    assert rel_l2(m32, o) < 1e-5
    assert rel_l2(m16, o) < 2e-3
    # the last input interval repeats the last sample (splineInterpolation's clamp)
    assert np.array_equal(m32[:, -factor:], np.repeat(m32[:, -factor:-factor + 1], factor, axis=1))


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


def test_gpu_echo_synthesis_matches_numpy(ctx):
    """Noise-free echoes synthesised on the device equal the numpy generator's (same
    Newton paths, same centred-chirp model) to 1e-9 relative."""
    spec = S.scaled(S.config_spec(2), n_pulses=16, n_samples=4096, n_scatterers=5, snr_db=np.inf)
    sc = S.make_scene(spec)
    sid = bsar.synthesize_scene(ctx, sc)
    try:
        raw = ctx.scene_read_samples(sid, spec.n_pulses, spec.n_samples)
    finally:
        ctx.scene_release(sid)
    assert rel_l2(raw, sc.raw) < 1e-9


def test_gpu_echo_synthesis_noise_statistics(ctx):
    spec = S.scaled(S.config_spec(1), n_pulses=64, n_scatterers=0, snr_db=10.0)
    sc = S.make_scene(spec, with_raw=False)
    sid = bsar.synthesize_scene(ctx, sc)
    try:
        raw = ctx.scene_read_samples(sid, spec.n_pulses, spec.n_samples)
    finally:
        ctx.scene_release(sid)
    nc = int(spec.pulse_T * spec.fs) + 1
    want = nc / 10.0                        # Nc / SNR
    got = np.mean(np.abs(raw) ** 2)
    assert abs(got / want - 1.0) < 0.02
    assert abs(np.mean(raw)) < 0.05 * np.sqrt(want)


def test_gpu_echo_synthesis_reference_bins(ctx):
    """BSAR_SYNTH_REFERENCE_BINS: the simulator's echo placement (delta at sample
    1 + round(t * fs), circular convolution with the fftshifted chirp,
    src/raw_data_processing.cpp:292-406) restated in numpy, to 1e-9."""
    spec = S.scaled(S.config_spec(1), n_pulses=12, n_samples=2048, n_scatterers=3, snr_db=np.inf)
    sc = S.make_scene(spec, with_raw=False)
    L = S.optical_paths(sc, sc.scat_pos)                       # (Np, S), FP64 Newton paths
    N = spec.n_samples
    chirp = S.make_chirp(spec)
    ref = S.matched_reference(chirp, N)
    aux = np.zeros((spec.n_pulses, N), complex)
    for p in range(spec.n_pulses):
        for s_ in range(len(sc.scat_amp)):
            b = 1 + int(np.floor(L[p, s_] / 3e8 * spec.fs + 0.5))
            if 0 <= b < N:
                aux[p, b] += sc.scat_amp[s_] * np.exp(-2j * np.pi * spec.fc * L[p, s_] / 3e8)
    want = np.fft.ifft(np.fft.fft(aux, axis=1) * np.fft.fft(ref)[None, :], axis=1)
    dem = bsar.DemArrays(sc.x_vec, sc.y_vec, sc.z)
    f0, f1 = -spec.bandwidth / 2, spec.bandwidth / 2
    sid = ctx.scene_synthesize(dem, sc.tx, sc.rx, N, sc.scat_pos, sc.scat_amp, upsample=spec.upsample, n1=spec.n1,
                               n2=spec.n2, c=3e8, fc=spec.fc, fs=spec.fs, chirp_f0=f0, chirp_f1=f1,
                               chirp_T=spec.pulse_T, reference_bins=True)
    try:
        got = ctx.scene_read_samples(sid, spec.n_pulses, N)
    finally:
        ctx.scene_release(sid)
    assert rel_l2(got, want) < 1e-9
