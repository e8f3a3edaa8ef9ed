"""Each kernel family on the GPU against the oracle, through the C ABI's
single-stage entry points. Exact form: bit-identical results, except the
dB conversion, whose natural log is CUDA's (1-ulp differences from glibc's
log are counted and bounded)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def audio0():
    from akvisqol_b200 import synth
    return synth.audio_pair(synth.SEED_BASE)


@pytest.mark.parametrize("nb,sr,frames", [(32, 48000, 3), (32, 48000, 41), (21, 16000, 37), (32, 44100, 9)])
def test_spectrogram_bit_identical(native, oracle, nb, sr, frames):
    high = 8000.0 if nb == 21 else sr / 2.0
    coeffs, _ = oracle.filters(nb, sr, 50.0, high)
    window, hop = oracle.window_hop(sr)
    rng = np.random.default_rng(nb * 1000 + frames)
    x = rng.uniform(-1, 1, window + (frames - 1) * hop + int(rng.integers(0, hop)))
    got = native.spectrogram(x, coeffs, oracle.hann(window), window, hop)
    want = oracle.spectrogram(x, coeffs, window, hop)
    assert got.shape == want.shape
    assert np.array_equal(got, want)


def test_spectrogram_full_pair(native, oracle, audio0):
    ref, _ = audio0
    coeffs, _ = oracle.filters(32, 48000)
    window, hop = oracle.window_hop(48000)
    got = native.spectrogram(ref, coeffs, oracle.hann(window), window, hop)
    want = oracle.spectrogram(ref, coeffs, window, hop)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("n", [1, 2, 4, 8, 64, 4096, 8192, 1 << 16, 1 << 17, 1 << 20])
def test_fft_bit_identical(native, oracle, n):
    rng = np.random.default_rng(n)
    x = rng.uniform(-0.5, 0.5, n) + 1j * rng.uniform(-0.5, 0.5, n)
    fwd = native.fft(x)
    assert np.array_equal(fwd.view(np.float64), oracle.fft_dif(x).view(np.float64))
    inv = native.fft(fwd, inverse=True)
    assert np.array_equal(inv.view(np.float64), oracle.fft_dit(fwd).view(np.float64))


def test_best_lag_reference_cases(native, kats):
    for c in kats["best_lag"]["cases"]:
        assert native.best_lag(c["ref"], c["deg"]) == c["lag"]


def test_lags_random(native, oracle):
    rng = np.random.default_rng(1)
    for _ in range(12):
        la, lb = int(rng.integers(1, 5000)), int(rng.integers(1, 5000))
        a = rng.uniform(-1, 1, la)
        b = np.concatenate([np.zeros(int(rng.integers(0, 50))), a])[:lb] + 0.05 * rng.standard_normal(lb)[:lb] \
            if lb <= la + 50 else rng.uniform(-1, 1, lb)
        assert native.best_lag(a, b) == oracle.best_lag(a, b)
        assert native.envelope_lag(a, b) == oracle.envelope_lag(a, b)


@pytest.mark.parametrize("columns", ["0", "1", "2"])
@pytest.mark.parametrize("rows_log2", [3, 4, 5, 6, 7, 8, 9, 10, 11])
def test_lags_column_pass_sizes(native, oracle, rows_log2, columns, monkeypatch):
    """Signal lengths whose transforms have 2^rows_log2 rows of 4096 points,
    with each column-pass implementation: shared-memory tiles (0) and, for
    4..11 rows_log2, registers (1) and registers with the forward pass's
    samples staged in shared memory (2)."""
    monkeypatch.setenv("VISQOL_LAG_COLUMNS", columns)
    n = 4096 << rows_log2
    rng = np.random.default_rng(100 + rows_log2)
    la = int(0.4 * n)
    a = rng.uniform(-1, 1, la)
    shift = int(rng.integers(1, 400))
    b = np.concatenate([np.zeros(shift), a])[:la + 57] + 0.05 * rng.standard_normal(la + 57)
    assert native.best_lag(a, b) == oracle.best_lag(a, b)
    assert native.envelope_lag(a, b) == oracle.envelope_lag(a, b)


def test_envelope_lag_full_pair(native, oracle, audio0):
    ref, deg = audio0
    assert native.envelope_lag(ref, deg) == oracle.envelope_lag(ref, deg)


def test_log10_agreement(native, oracle):
    rng = np.random.default_rng(9)
    x = 10.0 ** rng.uniform(-9, 1, 1 << 20)
    got = native.log10x10(x)
    want = oracle.convert_to_db(x, -1e300)
    diff = got != want
    ulps = np.abs(got.view(np.int64) - want.view(np.int64))
    print(f"log10 agreement: {1 - diff.mean():.6f} bit-identical, max {ulps.max()} ulp")
    # CUDA's natural log differs from glibc's by an ulp or two on rare inputs
    assert ulps.max() <= 2
    assert diff.mean() < 1e-2


def test_prepare_for_comparison(native, oracle, audio0):
    ref, deg = audio0
    coeffs, _ = oracle.filters(32, 48000)
    window, hop = oracle.window_hop(48000)
    rs = oracle.spectrogram(ref, coeffs, window, hop)
    ds = oracle.spectrogram(deg[1778:], coeffs, window, hop)
    gr, gd = native.prepare_for_comparison(rs, ds)
    wr, wd = oracle.prepare_for_comparison(rs, ds)
    # identical up to the rare one-ulp log differences
    assert np.max(np.abs(gr - wr)) < 1e-12 and np.max(np.abs(gd - wd)) < 1e-12
    assert (gr != wr).mean() < 1e-3 and (gd != wd).mean() < 1e-3


def test_nsim_table_bit_identical(native, oracle, audio0):
    ref, deg = audio0
    coeffs, _ = oracle.filters(32, 48000)
    window, hop = oracle.window_hop(48000)
    rs, ds = oracle.prepare_for_comparison(oracle.spectrogram(ref, coeffs, window, hop),
                                           oracle.spectrogram(deg[1778:], coeffs, window, hop))
    idx = oracle.ref_patch_indices(rs.shape[1], 30)
    nfd = ds.shape[1]
    keep = oracle.calc_max_num_patches(idx, nfd, 30)
    idx = idx[:keep]
    lo = np.maximum(0, idx - 1800)
    hi = np.maximum(lo, np.minimum(idx + 1800, nfd - 1))
    got = native.nsim_table(rs, ds, 30, idx, lo, hi)
    want = oracle.nsim_table(rs, ds, 30, idx, lo, hi)
    for p in range(idx.size):
        assert np.array_equal(got[p, lo[p]:hi[p] + 1], want[p, lo[p]:hi[p] + 1])


def test_nsim_table_small_windows(native, oracle):
    rng = np.random.default_rng(3)
    nb, patch, nfr, nfd = 21, 20, 160, 150
    rs = rng.uniform(0, 60, (nb, nfr))
    ds = rng.uniform(0, 60, (nb, nfd))
    idx = np.array([9, 29, 49, 69, 89, 109, 129])
    lo = np.maximum(0, idx - 40)
    hi = np.maximum(lo, np.minimum(idx + 40, nfd - 1))
    got = native.nsim_table(rs, ds, patch, idx, lo, hi)
    want = oracle.nsim_table(rs, ds, patch, idx, lo, hi)
    for p in range(idx.size):
        assert np.array_equal(got[p, lo[p]:hi[p] + 1], want[p, lo[p]:hi[p] + 1])


@pytest.mark.parametrize("seed", range(6))
def test_dp_identical(native, oracle, seed):
    rng = np.random.default_rng(seed)
    np_, nfd = int(rng.integers(1, 20)), int(rng.integers(20, 900))
    sims = rng.uniform(-0.2, 1.0, (np_, nfd))
    if seed % 2:
        sims = np.round(sims, 1)  # many exact ties
    idx = np.sort(rng.integers(0, nfd, np_))
    radius = int(rng.integers(1, 200))
    lo = np.maximum(0, idx - radius)
    hi = np.maximum(lo, np.minimum(idx + radius, nfd - 1))
    off, valid, reached = native.dp(sims, lo, hi)
    woff, wvalid, wreached = oracle.dp_backtrack(sims, lo, hi)
    assert reached == wreached
    assert np.array_equal(off, woff) and np.array_equal(valid, wvalid)


def test_dp_reference_case(native, oracle, kats):
    k = kats["dp_start_times"]
    ref = np.array(k["ref_rows"])
    deg = np.array(k["deg"]).reshape(k["num_bands"], k["nf_deg"])
    idx = np.array(k["indices"])
    lo = np.maximum(0, idx - 8)
    hi = np.maximum(lo, np.minimum(idx + 8, k["nf_deg"] - 1))
    sims = native.nsim_table(ref, deg, 1, idx, lo, hi)
    off, valid, _ = native.dp(sims, lo, hi)
    for p, want in k["expected"].items():
        assert (off[int(p)] if valid[int(p)] else 0.0) == want


@pytest.mark.parametrize("nr,nc", [(3, 1), (32, 30), (21, 20), (32, 27), (32, 2), (5, 4)])
def test_patch_similarity_bit_identical(native, oracle, nr, nc):
    rng = np.random.default_rng(nr * 100 + nc)
    ref = rng.uniform(0, 50, (nr, nc))
    deg = rng.uniform(0, 50, (nr, nc))
    gm, gmeans, gsd, gen = native.patch_similarity(ref, deg)
    wm, wmeans, wsd, wen = oracle.patch_similarity(ref, deg)
    assert gm == wm
    assert np.array_equal(gmeans, wmeans) and np.array_equal(gsd, wsd) and np.array_equal(gen, wen)


def test_fast_quotient_within_one_ulp(native):
    """The fast forms' NSIM quotient (reciprocal estimate refined by
    Markstein's Newton-Raphson steps, then one quotient correction) against
    IEEE division: within one ulp of n / d everywhere, over random operands
    spanning the table's range and edge denominators (powers of two, values
    one ulp from them, the NSIM constants and their products)."""
    rng = np.random.default_rng(11)
    m = 1 << 20
    num = rng.standard_normal(m) * np.exp(rng.uniform(-30, 30, m))
    den = np.exp(rng.uniform(-40, 40, m))
    c1, c3 = 1e-4, 4.5e-4
    edges = np.array([1.0, 2.0, 0.5, 2.0 ** 100, 2.0 ** -100, c1, c3, c3 * c3, c1 * c3, 3.0, 1.0 / 3.0,
                      np.nextafter(1.0, 2.0), np.nextafter(1.0, 0.0), np.nextafter(2.0, 0.0),
                      np.nextafter(2.0 ** 600, np.inf), 2.0 ** -1000, 2.0 ** 1000])
    en = np.repeat(rng.standard_normal(64), edges.size)
    ed = np.tile(edges, 64)
    num, den = np.concatenate([num, en, np.ones(edges.size)]), np.concatenate([den, ed, edges])
    got = native.nsim_quotient(num, den)
    want = num / den
    ulp = np.spacing(np.abs(want))
    err = np.abs(got - want) / ulp
    assert np.all(np.isfinite(got))
    assert float(err.max()) <= 1.0, float(err.max())
    assert float(np.mean(got == want)) > 0.99
