"""The oracle against the reference's own known-answer tests.

Every vector comes from tests/golden/reference_kats.json, extracted from the
reference's inline Zig tests (file:line in each entry's "cite")."""

import numpy as np
import pytest


def test_erb_center_freqs(oracle, kats):
    k = kats["erb_center_freqs"]
    cf = np.zeros(k["n"])
    oracle.lib.vqo_uniform_center_freqs(k["n"], k["low"], k["high"], oracle._d(cf))
    (first, tf), (last, tl) = k["first_last"]
    assert abs(cf[0] - first) <= tf
    assert abs(cf[-1] - last) <= tl
    assert np.all(np.diff(cf) < 0)


def test_filters_ascending_and_finite(oracle, kats):
    coeffs, cf = oracle.filters(32, 48000, 50.0, 24000.0)
    (first, tf), (last, tl) = kats["gammatone_center_freqs"]["first_last"]
    assert abs(cf[0] - first) <= tf and abs(cf[-1] - last) <= tl
    assert np.all(np.diff(cf) > 0)
    assert np.all(np.isfinite(coeffs)) and np.all(coeffs[:, 7] > 0)


def test_lowest_band_first_outputs(oracle, kats):
    k = kats["gammatone_lowest_band"]
    coeffs, _ = oracle.filters(32, 48000, 50.0, 24000.0)
    x = oracle.f64(k["samples"])
    out = np.zeros(x.size)
    oracle.lib.vqo_filter_band(oracle._d(oracle.f64(coeffs[0])), oracle._d(x), x.size, oracle._d(out))
    for i, (want, tol) in enumerate(k["expected"]):
        assert abs(out[i] - want) <= tol


def test_hann_symmetric():
    import oracle as O
    w = O.hann(16)
    assert abs(w[0]) < 1e-12 and abs(w[15]) < 1e-12
    assert np.allclose(w[:8], w[15:7:-1], atol=1e-12)


def test_db_reference_values(oracle, kats):
    k = kats["db_reference"]
    out = oracle.convert_to_db(k["data"], k["floor"])
    assert np.allclose(out, k["expected"], atol=k["tol"], rtol=0)
    k = kats["db_clamp"]
    out = oracle.convert_to_db(k["data"], k["floor"])
    assert np.allclose(out, k["expected"], atol=1e-9, rtol=0)


def test_joint_min_and_floor(oracle, kats):
    k = kats["joint_min"]
    a, b = oracle.f64(k["a"]).copy(), oracle.f64(k["b"]).copy()
    oracle.lib.vqo_subtract_joint_minimum(oracle._d(a), a.size, oracle._d(b), b.size)
    assert np.allclose(np.concatenate([a, b]), k["expected"], atol=1e-12, rtol=0)
    k = kats["floor_per_frame"]
    ref, deg = oracle.f64(k["ref"]).copy(), oracle.f64(k["deg"]).copy()
    oracle.lib.vqo_raise_floor_per_frame(oracle._d(ref), oracle._d(deg), 2, 2, 2, 45.0)
    assert np.allclose(np.concatenate([ref, deg]), k["expected"], atol=1e-12, rtol=0)


def test_prepare_for_comparison_floors(oracle):
    rng = np.random.default_rng(3)
    ref = rng.uniform(0, 1, (4, 9)) ** 4
    deg = rng.uniform(0, 1, (4, 7)) ** 4
    ref[1, 2] = 0.0
    r, d = oracle.prepare_for_comparison(ref, deg)
    assert min(r.min(), d.min()) == 0.0
    rdb = np.maximum(10 * np.log10(np.where(ref == 0, np.finfo(float).eps, ref)), -45)
    ddb = np.maximum(10 * np.log10(deg), -45)
    cols = min(9, 7)
    floor = np.maximum(rdb[:, :cols], ddb[:, :cols]).max(axis=0) - 45
    rdb[:, :cols] = np.maximum(rdb[:, :cols], floor)
    ddb[:, :cols] = np.maximum(ddb[:, :cols], floor)
    lo = min(rdb.min(), ddb.min())
    assert np.allclose(r, rdb - lo, atol=1e-9) and np.allclose(d, ddb - lo, atol=1e-9)


@pytest.mark.parametrize("case", range(5))
def test_best_lag_cases(oracle, kats, case):
    c = kats["best_lag"]["cases"][case]
    assert oracle.best_lag(c["ref"], c["deg"]) == c["lag"]


def test_fft_size_for(oracle, kats):
    for biggest, want in kats["fft_size_for"]["pairs"]:
        assert oracle.lib.vqo_fft_size_for(biggest) == want


def test_conv2d_reference(oracle, kats):
    k = kats["conv2d"]
    cols = np.array(k["cols"])            # [4][5] column-major
    x = cols.T.copy()                     # 5 x 4 row-major
    out = oracle.conv2d3x3(x)
    assert np.allclose(out, np.array(k["expected_cols"]).T, atol=k["tol"], rtol=0)


def test_patch_similarity_3x1(oracle, kats):
    k = kats["patch_similarity_3x1"]
    mean, means, sd, en = oracle.patch_similarity(np.array(k["ref"]).reshape(3, 1), np.array(k["deg"]).reshape(3, 1))
    assert np.allclose(means, k["expected_means"], atol=k["tol"], rtol=0)


def test_identical_patches_score_one(oracle):
    sig = np.sin(np.arange(20) * 0.3) + 1.5
    assert abs(oracle.similarity_scalar(sig.reshape(4, 5), sig.reshape(4, 5)) - 1.0) < 1e-9


def test_ref_patch_indices(oracle, kats):
    k = kats["ref_patch_indices"]
    assert list(oracle.ref_patch_indices(k["num_frames"], k["patch"])) == k["expected"]


def test_calc_max_num_patches(oracle, kats):
    k = kats["calc_max_num_patches"]
    for nf_deg, patch, want in k["cases"]:
        assert oracle.calc_max_num_patches(k["idx"], nf_deg, patch) == want


def test_dp_start_times(oracle, kats):
    k = kats["dp_start_times"]
    ref = np.array(k["ref_rows"])
    deg = np.array(k["deg"]).reshape(k["num_bands"], k["nf_deg"])
    nfd, radius, patch = k["nf_deg"], k["radius"], k["patch"]
    idx = np.array(k["indices"])
    lo = np.maximum(0, idx - radius * patch)
    hi = np.maximum(lo, np.minimum(idx + radius * patch, nfd - 1))
    sims = oracle.nsim_table(ref, deg, patch, idx, lo, hi)
    off, valid, _ = oracle.dp_backtrack(sims, lo, hi)
    for p, want in k["expected"].items():
        # deg_patch_start_time: offset * frame duration, 0 for an invalid match (src/dp.zig:335-345)
        t = off[int(p)] * k["frame_duration"] if valid[int(p)] else 0.0
        assert t == pytest.approx(want, abs=1e-9)


def test_slices(oracle, kats):
    k = kats["slice_in_range"]
    pad, base, n = oracle.slice_layout(len(k["signal"]), k["sr"], k["t0"], k["t1"])
    assert pad + n == k["len"] and k["signal"][base] == k["first"] and k["signal"][base + n - 1] == k["last"]
    k = kats["slice_padded"]
    pad, base, n = oracle.slice_layout(k["len"], k["sr"], k["t0"], k["t1"])
    assert pad + n == k["out_len"]
    assert pad + (k["one_at"] - base) == k["one_out_at"]


def test_lag_samples_back(oracle, kats):
    k = kats["lag_samples_back"]
    ln, ro, do, ls = oracle.trim_geometry(1000, 2000, k["lag"], k["sr"])
    assert ro == k["expected"]


def test_vad_first_patch(oracle, kats):
    k = kats["vad"]
    sig = np.zeros(k["len"])
    n = np.arange(k["active"][0], k["active"][1])
    sig[n] = np.sin(n * k["freq_per_sample"])
    nf = 1 + (sig.size - k["window"]) // (k["window"] // 4)
    idx = oracle.vad_patch_indices(sig, nf, k["patch"], k["window"], k["overlap"])
    assert len(idx) >= 2 and len(idx) < (nf - 9) // 20
    assert idx[0] == k["first"]


def test_spl_unit_dc(oracle, kats):
    want, tol = kats["spl_unit_dc"]["expected"]
    assert abs(oracle.spl(np.ones(16)) - want) <= tol


def test_svr_manual_and_default(oracle, kats):
    k = kats["svr_manual_rbf"]
    assert abs(oracle.svr_predict(k["obs"], k["model"]) - k["expected"][0]) <= k["expected"][1]
    k = kats["svr_default_known"]
    assert abs(oracle.svr_predict(k["obs"]) - k["expected"][0]) <= k["expected"][1]
