"""The FP32 form's lag search against the exact search and the oracle.

The f32 transform only nominates: every lag whose |Re| lies within twice the
f32 error bound of the largest is rescored by f64 dot products, and the
first maximum in ascending lag wins (reference refineLag / rescore,
src/xcorr.zig:270-340; GPU flow src/gpu/engine.zig:445-540). The lag must
equal the exact search's on every input; with more than 64 candidates the
exact search decides.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS32 = float(np.finfo(np.float32).eps)


def fft_size(m: int) -> int:
    n = 1
    while n < 2 * m - 1:
        n <<= 1
    return n


def circular_xcorr(a, b, n):
    """sum_t a[t + i] b[t], circular index i, in f64 (numpy's FFT)."""
    fa = np.fft.fft(np.concatenate([a, np.zeros(n - a.size)]))
    fb = np.fft.fft(np.concatenate([b, np.zeros(n - b.size)]))
    return np.fft.ifft(fa * np.conj(fb)).real


@pytest.mark.parametrize("length", [37, 500, 4096])
def test_refine_lag_kat(native, oracle, length):
    """The reference's refineLag case (src/xcorr.zig:403-429): s1 uniform in
    [0.5, 1.5), s2 = s1 delayed by 9 with uniform noise around it, 13 samples
    longer; the correlation perturbed by up to tol (|s1|^2 + |s2|^2) with
    tol = 1e-6 and rounded to f32. The device nomination and rescoring must
    return bestLag's answer."""
    rng = np.random.default_rng(7 + length)
    s1 = rng.random(length) + 0.5
    s2 = rng.random(length + 13)
    s2[9:9 + length] = s1
    want = oracle.best_lag(s1, s2)
    n = fft_size(s2.size)
    e = float(np.sum(s1 * s1) + np.sum(s2 * s2))
    tol = 1e-6
    approx = (circular_xcorr(s1, s2, n) + (rng.random(n) * 2 - 1) * tol * e).astype(np.float32)
    assert native.refine_lag(s1, s2, approx, 1.0, tol) == want


def test_refine_lag_gives_up_over_64_candidates(native):
    """A flat correlation (constant signals, a large tolerance): more than 64
    lags qualify and the search reports no lag, as refineLag returns null."""
    s1 = np.ones(300)
    s2 = np.ones(300)
    n = fft_size(300)
    approx = circular_xcorr(s1, s2, n).astype(np.float32)
    assert native.refine_lag(s1, s2, approx, 1.0, 0.5) is None


@pytest.mark.parametrize("length", [1500, 3000, 9000, 30000, 120000, 480000])
def test_f32_correlation_within_bound(native, oracle, length):
    """The f32 correlation's error stays far inside the bound the nomination
    assumes, tol(n) n (|a|^2 + |b|^2) with tol(n) = 8 eps_f32 log2(n)
    (src/gpu/engine.zig:820-822): the ratio is asserted below 1/4 of it.
    Envelopes of audio-like signals, transform sizes from 4096 (one CTA) to
    2^20 (the three-pass search with register column passes)."""
    from akvisqol_b200 import synth
    ref, deg = synth.audio_pair(synth.SEED_BASE + 50, seconds=length / 48000.0 + 0.2)
    delay = int(round(0.037 * 48000))  # the degraded signal's leading silence
    a, b = ref[:length], deg[delay:delay + length + length // 7]
    lag, undecided, corr = native.lag_search(a, b, form="fast", corr=True)
    n = corr.size
    ea, eb = oracle.upper_envelope(a), oracle.upper_envelope(b)
    exact = n * circular_xcorr(ea, eb, n)
    err = float(np.max(np.abs(corr.astype(np.float64) - exact)))
    bound = 8 * EPS32 * np.log2(n) * n * float(np.sum(ea * ea) + np.sum(eb * eb))
    assert err <= 0.25 * bound, (err / bound)
    assert undecided == 0
    assert lag == oracle.envelope_lag(a, b)


def _pairs(seed, count, lo, hi):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        la, lb = int(rng.integers(lo, hi)), int(rng.integers(lo, hi))
        a = rng.standard_normal(la)
        shift = int(rng.integers(0, max(1, min(la, lb) // 3)))
        b = 0.05 * rng.standard_normal(lb)
        m = min(la, lb - shift)
        if m > 0:
            b[shift:shift + m] += a[:m]
        if rng.random() < 0.5:
            a, b = b, a
        out.append((a, b))
    return out


@pytest.mark.parametrize("raw", [True, False])
@pytest.mark.parametrize("lo,hi", [(30, 2000), (3000, 16000), (20000, 200000)])
def test_fast_lags_equal_exact(native, oracle, raw, lo, hi):
    """Random pairs (a shifted noisy copy, either order) at sizes that take
    every form of the search: one CTA (n <= 4096), shared-memory column
    passes (8192 .. 32768), register column passes (2^16 ..)."""
    for a, b in _pairs(1000 * lo + raw, 6, lo, hi):
        want = oracle.best_lag(a, b) if raw else oracle.envelope_lag(a, b)
        lag, undecided, _ = native.lag_search(a, b, raw=raw, form="fast")
        assert lag == want, (a.size, b.size, lag, want, undecided)
        assert native.lag_search(a, b, raw=raw, form="exact")[0] == want


@pytest.mark.parametrize("kind", ["silence", "constant", "periodic"])
def test_fast_lag_undecided_falls_back(native, oracle, kind):
    """Inputs with runs of equal correlation: over 64 candidates (silence,
    constants), or equal peaks that only rounding orders (a periodic
    signal's lags one period apart): the f32 search leaves the lag to the
    exact search, whose answer (the CPU's first maximum) is returned."""
    n = 20000
    if kind == "silence":
        a, b = np.zeros(n), np.zeros(n + 100)
    elif kind == "constant":
        a, b = np.full(n, 0.25), np.full(n + 100, 0.25)
    else:
        t = np.arange(n + 100)
        b = np.sin(2 * np.pi * t / 50.0)
        a = b[:n].copy()
    for raw in (True, False):
        want = oracle.best_lag(a, b) if raw else oracle.envelope_lag(a, b)
        lag, undecided, _ = native.lag_search(a, b, raw=raw, form="fast")
        assert lag == want, (kind, raw, lag, want)
        assert undecided == 1


@pytest.mark.parametrize("columns", ["0", "1", "2"])
@pytest.mark.parametrize("rows_log2", [1, 3, 4, 6, 8, 9, 11])
def test_fast_lags_column_pass_shapes(native, oracle, rows_log2, columns, monkeypatch):
    """The f32 search with each column-pass shape (shared-memory tiles;
    registers; registers with the forward samples staged) at transforms of
    2^rows_log2 rows of 4096 points: the exact search's lag."""
    monkeypatch.setenv("VISQOL_LAG_COLUMNS", columns)
    n = 4096 << rows_log2
    rng = np.random.default_rng(300 + rows_log2)
    la = int(0.4 * n)
    a = rng.uniform(-1, 1, la)
    shift = int(rng.integers(1, 400))
    b = np.concatenate([np.zeros(shift), a])[:la + 57] + 0.05 * rng.standard_normal(la + 57)
    for raw in (True, False):
        want = oracle.best_lag(a, b) if raw else oracle.envelope_lag(a, b)
        assert native.lag_search(a, b, raw=raw, form="fast")[0] == want
