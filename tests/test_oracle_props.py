"""Oracle self-consistency: the properties the reference's own tests assert
(bit-identity of its fast paths to their scalar definitions, FFT round
trips, trim geometry vs truncation), checked on the oracle's restatement."""

import numpy as np
import pytest


def test_spectrogram_lanes_equal_scalar(oracle):
    # reference src/gammatone.zig:579-610: frame count not a multiple of the lane width
    coeffs, _ = oracle.filters(32, 48000)
    window, hop, nf = 384, 96, 3 * 8 + 1
    rng = np.random.default_rng(0x9A77)
    sig = rng.uniform(-1, 1, window + (nf - 1) * hop)
    spec = oracle.spectrogram(sig, coeffs, window, hop)
    hann = oracle.hann(window)
    for f in range(nf):
        frame = oracle.f64(sig[f * hop:f * hop + window] * hann)
        for b in (0, 7, 31):
            want = oracle.lib.vqo_filter_band_rms_fresh(oracle._d(oracle.f64(coeffs[b])), oracle._d(frame), window)
            assert spec[b, f] == want


def test_spectrogram_shape_finite(oracle):
    coeffs, _ = oracle.filters(32, 48000)
    window, hop = oracle.window_hop(48000)
    rng = np.random.default_rng(0xABC123)
    sig = rng.uniform(-1, 1, window * 4 + hop * 7)
    spec = oracle.spectrogram(sig, coeffs, window, hop)
    assert spec.shape == (32, 1 + (sig.size - window) // hop)
    assert np.all(np.isfinite(spec)) and np.all(spec >= 0)


def test_similarity_at_equals_scalar(oracle):
    # reference src/nsim.zig:606-638: the plane-reusing path is bit-identical
    nr, nc, nf = 6, 5, 17
    rng = np.random.default_rng(0x5EED)
    spec = rng.uniform(0, 40, (nr, nf))
    ref = rng.uniform(0, 40, (nr, nc))
    # The table holds offsets 0..nf-1; windows past the end read zeros.
    table = oracle.nsim_table(ref, spec, nc, [0], [0], [nf - 1])
    for off in range(nf):
        deg = np.zeros((nr, nc))
        for c in range(nc):
            if off + c < nf:
                deg[:, c] = spec[:, off + c]
        assert table[0, off] == oracle.similarity_scalar(ref, deg)


@pytest.mark.parametrize("n", [2, 4, 8, 32, 1 << 13, 1 << 15])
def test_dif_matches_natural_fft(oracle, n):
    rng = np.random.default_rng(7)
    x = rng.uniform(-0.5, 0.5, n) + 1j * rng.uniform(-0.5, 0.5, n)
    y = oracle.fft_dif(x)
    bits = int(np.log2(n))
    br = np.array([int(format(i, f"0{bits}b")[::-1], 2) for i in range(n)])
    ref = np.fft.fft(x)[br]
    assert np.allclose(y, ref, atol=1e-9 * n, rtol=0)
    z = oracle.fft_dit(y) / n
    assert np.allclose(z, x, atol=1e-12, rtol=0)


def test_best_lag_matches_direct_xcorr(oracle):
    # reference src/xcorr.zig:383-401: fast path == three-FFT reference
    rng = np.random.default_rng(1)
    for _ in range(20):
        l1, l2 = 50 + rng.integers(0, 3000), 50 + rng.integers(0, 3000)
        a = rng.uniform(-1, 1, l1)
        shift = int(rng.integers(0, 40))
        b = np.where((np.arange(l2) >= shift) & (np.arange(l2) - shift < l1),
                     np.concatenate([np.zeros(shift), a, np.zeros(max(0, l2))])[:l2] + 0.1 * (rng.random(l2) - 0.5),
                     0.05 * rng.random(l2))
        big = max(l1, l2)
        full = np.correlate(np.pad(a, (0, big - l1)), np.pad(b, (0, big - l2)), "full")  # lags -(big-1)..(big-1)
        lags = np.arange(-(big - 1), big)
        want = lags[np.argmax(np.abs(full))]
        assert oracle.best_lag(a, b) == -want or oracle.best_lag(a, b) == want


def test_envelope_properties(oracle):
    # reference src/envelope.zig:55-86
    assert np.allclose(oracle.upper_envelope(np.zeros(8)), 1e-6, atol=1e-12)
    assert np.allclose(oracle.upper_envelope(np.full(16, 0.7)), 0.7 + 1e-6, atol=1e-12)
    env = oracle.upper_envelope(np.sin(2 * np.pi * 4 * np.arange(128) / 128))
    assert np.all(np.isfinite(env)) and np.any(env > 1e-3)


def test_trim_geometry_equals_truncation(oracle):
    # reference src/realign.zig:496-529
    rng = np.random.default_rng(5)
    for it in range(600):
        sr = (16000, 44100, 48000)[it % 3]
        rl, dl = int(rng.integers(0, 401)), int(rng.integers(0, 401))
        lag = {0: 27, 1: -55}.get(it % 4, int(rng.integers(-rl, rl + 1)) if rl else 0)
        ref = np.arange(1, rl + 1, dtype=float)
        deg = -np.arange(1, dl + 1, dtype=float)
        tr, td = oracle.truncate_aligned(ref, deg, lag, sr)
        ln, ro, do, ls = oracle.trim_geometry(rl, dl, lag, sr)
        assert tr.size == ln and td.size == ln
        for i in range(ln):
            assert tr[i] == ref[ro + i]
            j = do + i
            assert td[i] == (deg[j] if 0 <= j < dl else 0.0)


def test_zig_pow_matches_known(oracle):
    # pow(2, 1.5) by the Go/Zig method: 2 * exp(0.5 * log 2)
    import math
    assert oracle.zig_pow(2.0, 1.5) == math.ldexp(math.exp(0.5 * math.log(2.0)) * 0.5, 2)
    assert oracle.zig_pow(10.0, 0.0) == 1.0
    assert abs(oracle.zig_pow(10.0, -0.3) - 10 ** -0.3) < 1e-15


def test_measure_rejects_short_and_empty(oracle):
    with pytest.raises(oracle.OracleError) as e:
        oracle.measure(np.zeros(100), np.zeros(100), 48000)
    assert e.value.code == -5
    with pytest.raises(oracle.OracleError) as e:
        oracle.measure(np.zeros(0), np.zeros(0), 48000)
    assert e.value.code == -5
    with pytest.raises(oracle.OracleError) as e:
        oracle.measure(np.ones(10000), np.ones(10000), 0)
    assert e.value.code == -1


def test_batch_equals_single(oracle):
    from akvisqol_b200 import synth
    pairs = [synth.audio_pair(synth.SEED_BASE + i, seconds=3.0) for i in range(3)]
    batch = oracle.measure_batch([p[0] for p in pairs], [p[1] for p in pairs], 48000, threads=3)
    for (r, d), (code, res) in zip(pairs, batch):
        single, _ = oracle.measure(r, d, 48000, trace=False)
        assert code == 0 and res["moslqo"] == single["moslqo"]
