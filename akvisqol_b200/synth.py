"""Seeded synthetic audio pairs in the shapes of the ViSQOL workloads.

The reference benchmarks on conformance WAV files that are not available
here; these generators stand in for them with the same sample rates,
lengths, and kinds of degradation. Every pair is a pure function of its
seed (numpy PCG64), so the CPU model and the GPU see identical inputs.

* ``audio_pair``: 48 kHz music-like reference, pink noise at -20 dBFS plus
  six sinusoids (log-uniform 100 Hz-12 kHz, random phase) under a 4 Hz
  raised-cosine envelope. Degraded: 4th-order Butterworth lowpass (bilinear,
  f64), white noise at a given SNR, a delay of zeros prepended (the tail is
  kept, so the degraded signal is longer by the delay), int16 requantisation.
* ``speech_pair``: 16 kHz speech-like reference, a glottal pulse train with
  f0 drifting 100-220 Hz through three time-varying formant resonators, in
  0.3-1.2 s voiced runs separated by 0.1-0.5 s silences (so a VAD drops
  patches). Degraded: 8-bit mu-law round trip, 20 ms delay, 3% of 20 ms
  frames zeroed.
"""

from __future__ import annotations

import numpy as np
from scipy import signal as sps

SEED_BASE = 0x5EED_0000


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def _pink(rng: np.random.Generator, n: int) -> np.ndarray:
    """1/f noise by spectral shaping of white Gaussian noise."""
    white = rng.standard_normal(n)
    spec = np.fft.rfft(white)
    f = np.arange(spec.size, dtype=np.float64)
    f[0] = 1.0
    spec /= np.sqrt(f)
    spec[0] = 0.0
    x = np.fft.irfft(spec, n)
    return x / np.sqrt(np.mean(x * x))


def _requantise16(x: np.ndarray) -> np.ndarray:
    return np.clip(np.round(x * 32768.0), -32768, 32767) / 32768.0


def audio_pair(seed: int, seconds: float = 10.0, sample_rate: int = 48000, cutoff_hz: float = 12000.0,
               snr_db: float = 30.0, delay_s: float = 0.037) -> tuple[np.ndarray, np.ndarray]:
    """(reference, degraded) audio-mode pair; see the module docstring."""
    rng = _rng(seed)
    n = int(round(seconds * sample_rate))
    t = np.arange(n, dtype=np.float64) / sample_rate
    ref = 0.1 * _pink(rng, n)  # -20 dBFS RMS
    freqs = np.exp(rng.uniform(np.log(100.0), np.log(12000.0), 6))
    phases = rng.uniform(0.0, 2.0 * np.pi, 6)
    env = 0.5 - 0.5 * np.cos(2.0 * np.pi * 4.0 * t)
    tones = sum(0.08 * np.sin(2.0 * np.pi * f * t + p) for f, p in zip(freqs, phases))
    ref = ref + env * tones
    b, a = sps.butter(4, min(cutoff_hz, 0.49 * sample_rate), btype="low", fs=sample_rate)
    deg = sps.lfilter(b, a, ref)
    noise = rng.standard_normal(n)
    deg = deg + noise * (np.sqrt(np.mean(deg * deg)) * 10.0 ** (-snr_db / 20.0))
    delay = int(round(delay_s * sample_rate))
    deg = np.concatenate([np.zeros(delay), deg])
    return ref, _requantise16(deg)


def speech_pair(seed: int, seconds: float = 8.0, sample_rate: int = 16000,
                delay_s: float = 0.020, drop_fraction: float = 0.03) -> tuple[np.ndarray, np.ndarray]:
    """(reference, degraded) speech-mode pair; see the module docstring."""
    rng = _rng(seed)
    n = int(round(seconds * sample_rate))
    voiced = np.zeros(n, dtype=bool)
    pos = int(rng.uniform(0.05, 0.3) * sample_rate)
    while pos < n:
        run = int(rng.uniform(0.3, 1.2) * sample_rate)
        voiced[pos:pos + run] = True
        pos += run + int(rng.uniform(0.1, 0.5) * sample_rate)
    # glottal pulses with drifting f0
    t = np.arange(n) / sample_rate
    f0 = 100.0 + 120.0 * (0.5 + 0.5 * np.sin(2.0 * np.pi * rng.uniform(0.1, 0.4) * t + rng.uniform(0, 6.28)))
    phase = np.cumsum(f0 / sample_rate)
    pulses = (np.diff(np.floor(phase), prepend=0.0) > 0).astype(np.float64)
    src = sps.lfilter([1.0], [1.0, -1.8, 0.81], pulses)  # glottal spectral tilt
    src *= voiced
    # three formants, piecewise constant over 10 ms blocks
    block = sample_rate // 100
    ranges = [(300.0, 800.0), (900.0, 2500.0), (2500.0, 3500.0)]
    tracks = []
    for lo, hi in ranges:
        knots = rng.uniform(lo, hi, int(seconds * 4) + 2)
        tracks.append(np.interp(np.arange(0, n, block) / sample_rate, np.linspace(0, seconds, knots.size), knots))
    out = np.zeros(n)
    for k, (lo, hi) in enumerate(ranges):
        zi = np.zeros(2)
        bw = 80.0 + 40.0 * k
        y = np.zeros(n)
        for bi, start in enumerate(range(0, n, block)):
            f = tracks[k][bi]
            r = np.exp(-np.pi * bw / sample_rate)
            a = [1.0, -2.0 * r * np.cos(2.0 * np.pi * f / sample_rate), r * r]
            seg, zi = sps.lfilter([1.0 - r], a, src[start:start + block], zi=zi)
            y[start:start + block] = seg
        out += y * (1.0 / (k + 1))
    ref = 0.3 * out / (np.max(np.abs(out)) + 1e-12)
    # mu-law 8-bit round trip
    mu = 255.0
    c = np.sign(ref) * np.log1p(mu * np.abs(ref)) / np.log1p(mu)
    q = np.round((c + 1.0) * 127.5) / 127.5 - 1.0
    deg = np.sign(q) * ((1.0 + mu) ** np.abs(q) - 1.0) / mu
    frame = int(0.02 * sample_rate)
    frames = n // frame
    drop = rng.choice(frames, size=max(1, int(round(drop_fraction * frames))), replace=False)
    for fidx in drop:
        deg[fidx * frame:(fidx + 1) * frame] = 0.0
    deg = np.concatenate([np.zeros(int(round(delay_s * sample_rate))), deg])
    return ref, deg


def audio_batch(count: int, seed0: int = SEED_BASE, min_s: float = 3.0, max_s: float = 30.0):
    """Uneven audio pairs: log-uniform lengths, cutoff U(4, 16) kHz, SNR U(10, 40) dB, delay U(0, 200) ms."""
    return audio_batch_items(range(count), seed0, min_s, max_s)


def audio_batch_items(indices, seed0: int = SEED_BASE, min_s: float = 3.0, max_s: float = 30.0):
    """Items `indices` of audio_batch(count, seed0, min_s, max_s), for any count above them."""
    pairs = []
    for i in indices:
        r = _rng(seed0 + 0x10000 + i)
        secs = float(np.exp(r.uniform(np.log(min_s), np.log(max_s))))
        pairs.append(audio_pair(seed0 + i, seconds=secs, cutoff_hz=r.uniform(4000, 16000),
                                snr_db=r.uniform(10, 40), delay_s=r.uniform(0.0, 0.2)))
    return pairs


def speech_batch(count: int, seed0: int = SEED_BASE + 0x8000, min_s: float = 2.0, max_s: float = 15.0):
    pairs = []
    for i in range(count):
        r = _rng(seed0 + 0x10000 + i)
        pairs.append(speech_pair(seed0 + i, seconds=float(np.exp(r.uniform(np.log(min_s), np.log(max_s))))))
    return pairs
