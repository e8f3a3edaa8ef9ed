"""The product's host-side model (filter design, planning, SPL, SVR, WAV)
against the oracle, and the lanes' chunk planning against its rule, on the CPU: compiled from akvisqol_b200/csrc/host_model.cpp
into a test library with a thin C shim (tests/native/host_shim.cpp)."""

import ctypes
import math
import struct
import subprocess
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_size_t, c_uint32
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SHIM_SRC = ROOT / "tests" / "native" / "host_shim.cpp"
SHIM = ROOT / "tests" / "native" / "build" / "libhost_shim.so"


@pytest.fixture(scope="module")
def hs():
    SHIM.parent.mkdir(parents=True, exist_ok=True)
    csrc = ROOT / "akvisqol_b200" / "csrc"
    srcs = [SHIM_SRC, csrc / "host_model.cpp", csrc / "lattice.cpp", csrc / "tflite.cpp"]
    if not SHIM.is_file() or any(s.stat().st_mtime > SHIM.stat().st_mtime for s in srcs):
        model = ROOT / "akvisqol_b200" / "model" / "libsvm_nu_svr_model.txt"
        lattice = next((ROOT / "akvisqol_b200" / "model").glob("lattice_*.tflite"))
        subprocess.run(["g++", "-std=c++17", "-O2", "-march=x86-64-v3", "-fPIC", "-shared", "-ffp-contract=off",
                        "-fno-fast-math", "-I/usr/local/cuda/include", f"-DVQB_MODEL_PATH={model}",
                        f"-DVQB_LATTICE_PATH={lattice}", "-o", str(SHIM)]
                       + [str(s) for s in srcs], check=True)
    lib = ctypes.CDLL(str(SHIM))
    D, I64, SZ = POINTER(c_double), POINTER(c_int64), POINTER(c_size_t)
    for name, res, args in [
        ("hs_filterbank", None, [c_size_t, c_uint32, c_double, c_double, D, D, D]),
        ("hs_hann", None, [c_size_t, D]),
        ("hs_twiddles", None, [c_size_t, D]),
        ("hs_zig_pow", c_double, [c_double, c_double]),
        ("hs_geometry", None, [c_uint32, SZ, SZ, D]),
        ("hs_ref_patch_indices", c_int, [c_size_t, c_size_t, I64, SZ]),
        ("hs_vad", None, [D, c_size_t, c_size_t, c_size_t, c_size_t, c_double, I64, SZ]),
        ("hs_plan_search", c_int, [I64, c_size_t, c_size_t, c_size_t, c_size_t, c_int32, I64, I64, SZ]),
        ("hs_slice_layout", None, [c_size_t, c_uint32, c_double, c_double, I64, I64, I64]),
        ("hs_trim_geometry", None, [c_int64, c_int64, c_int64, c_uint32, I64, I64, I64, D]),
        ("hs_reuse_frame", c_int64, [c_int64, c_int64, c_int64, c_int64, c_size_t, c_size_t, c_size_t]),
        ("hs_spl_factor", c_double, [c_double, c_size_t, c_double, c_size_t]),
        ("hs_svr_predict", c_int, [c_char_p, c_size_t, D, D]),
        ("hs_decode_wav", c_int64, [c_char_p, c_size_t, D, c_size_t, POINTER(c_uint32)]),
        ("hs_chunk_bounds", c_size_t, [SZ, c_size_t, c_size_t, c_size_t, c_size_t, SZ]),
    ]:
        fn = getattr(lib, name)
        fn.restype, fn.argtypes = res, args
    return lib


def d(a):
    return a.ctypes.data_as(POINTER(c_double))


def i64(a):
    return a.ctypes.data_as(POINTER(c_int64))


@pytest.mark.parametrize("nb,sr,high", [(32, 48000, 24000.0), (21, 16000, 8000.0), (32, 44100, 22050.0)])
def test_filterbank_bit_identical(hs, oracle, nb, sr, high):
    coeffs, cf, run = np.zeros(8 * nb), np.zeros(nb), np.zeros(8 * nb)
    hs.hs_filterbank(nb, sr, 50.0, high, d(coeffs), d(cf), d(run))
    oc, ocf = oracle.filters(nb, sr, 50.0, high)
    assert np.array_equal(coeffs.reshape(nb, 8), oc)
    assert np.array_equal(cf, ocf)
    # filterBandRmsFresh's derived coefficients (reference src/gammatone.zig:269-277)
    r = run.reshape(nb, 8)
    gi = 1.0 / oc[:, 7]
    assert np.array_equal(r[:, 0], oc[:, 0] * gi) and np.array_equal(r[:, 1], oc[:, 1] * gi)
    assert np.array_equal(r[:, 6], oc[:, 5]) and np.array_equal(r[:, 7], oc[:, 6])


@pytest.mark.parametrize("size", [1, 2, 16, 1280, 3840])
def test_hann_bit_identical(hs, oracle, size):
    w = np.zeros(size)
    hs.hs_hann(size, d(w))
    assert np.array_equal(w, oracle.hann(size))


@pytest.mark.parametrize("n", [2, 64, 4096, 1 << 16])
def test_twiddles_bit_identical(hs, oracle, n):
    t = np.zeros(n)
    hs.hs_twiddles(n, d(t))
    o = np.zeros(n)
    oracle.lib.vqo_fft_twiddles(n, oracle._d(o))
    assert np.array_equal(t, o)


def test_zig_pow(hs, oracle):
    rng = np.random.default_rng(2)
    for y in list(rng.uniform(-3, 3, 200)) + [1.5, 0.5, -0.5, 0.0, 1.0, 2.0]:
        assert hs.hs_zig_pow(10.0, y) == oracle.zig_pow(10.0, y)
    assert hs.hs_zig_pow(2.0, 1.5) == oracle.zig_pow(2.0, 1.5)


@pytest.mark.parametrize("sr", [8000, 16000, 44100, 48000, 96000])
def test_geometry(hs, oracle, sr):
    w, h, fd = c_size_t(), c_size_t(), c_double()
    hs.hs_geometry(sr, ctypes.byref(w), ctypes.byref(h), ctypes.byref(fd))
    assert (w.value, h.value) == oracle.window_hop(sr)
    assert fd.value == h.value / sr


@pytest.mark.parametrize("nf,patch", [(200, 30), (497, 30), (397, 20), (45, 30), (44, 30), (30, 20)])
def test_ref_patch_indices(hs, oracle, nf, patch):
    out, n = np.zeros(nf, np.int64), c_size_t()
    rc = hs.hs_ref_patch_indices(nf, patch, i64(out), ctypes.byref(n))
    try:
        want = list(oracle.ref_patch_indices(nf, patch))
        assert rc == 0 and list(out[: n.value]) == want
    except oracle.OracleError:
        assert rc == -5


def test_vad_matches_oracle(hs, oracle):
    from akvisqol_b200 import synth
    for seed in range(4):
        ref, _ = synth.speech_pair(synth.SEED_BASE + seed, seconds=4.0 + 2 * seed)
        window, hop = oracle.window_hop(16000)
        nf = 1 + (ref.size - window) // hop
        out, n = np.zeros(nf, np.int64), c_size_t()
        hs.hs_vad(d(ref), ref.size, nf, 20, window, 0.25, i64(out), ctypes.byref(n))
        assert list(out[: n.value]) == list(oracle.vad_patch_indices(ref, nf, 20, window))


def test_plan_search_windows(hs, oracle):
    idx = np.array([14, 44, 74, 104, 134, 164, 194], np.int64)
    for nfr, nfd, radius in [(230, 230, 60), (230, 150, 2), (230, 180, 1), (230, 5, 60), (200, 230, 60)]:
        lo, hi, n = np.zeros(7, np.int64), np.zeros(7, np.int64), c_size_t()
        rc = hs.hs_plan_search(i64(idx), 7, nfr, nfd, 30, radius, i64(lo), i64(hi), ctypes.byref(n))
        keep = oracle.calc_max_num_patches(idx, nfd, 30)
        if keep == 0 or idx[keep - 1] + 30 > nfr:
            assert rc == -5  # SignalsTooDifferent (reference src/dp.zig:153-160)
            continue
        assert rc == 0 and n.value == keep
        sw = radius * 30
        want_lo = np.maximum(0, idx[:keep] - sw)
        want_hi = np.maximum(want_lo, np.minimum(idx[:keep] + sw, nfd - 1))
        assert np.array_equal(lo[:keep], want_lo) and np.array_equal(hi[:keep], want_hi)


def test_slice_layout_and_trim(hs, oracle):
    rng = np.random.default_rng(11)
    for _ in range(2000):
        sr = int(rng.choice([16000, 44100, 48000]))
        length = int(rng.integers(0, 500000))
        t0 = float(rng.uniform(-1.0, 12.0))
        t1 = t0 + float(rng.uniform(0.0, 1.0))
        a = [c_int64() for _ in range(3)]
        hs.hs_slice_layout(length, sr, t0, t1, *[ctypes.byref(x) for x in a])
        assert tuple(x.value for x in a) == oracle.slice_layout(length, sr, t0, t1)
        rl, dl = int(rng.integers(0, 60000)), int(rng.integers(0, 60000))
        lag = int(rng.integers(-rl - 5, rl + 5))
        b = [c_int64() for _ in range(3)] + [c_double()]
        hs.hs_trim_geometry(rl, dl, lag, sr, *[ctypes.byref(x) for x in b])
        assert tuple(x.value for x in b) == oracle.trim_geometry(rl, dl, lag, sr)


def test_reuse_frame_rule(hs):
    # RawSpectrograms.reuse (reference src/realign.zig:262-281)
    assert hs.hs_reuse_frame(0, 960 * 14, 28800, 0, 960, 27, 497) == 14
    assert hs.hs_reuse_frame(0, 960 * 14 - 1, 28800, 0, 960, 27, 497) == -1
    assert hs.hs_reuse_frame(10, 0, 100, 5, 960, 27, 497) == -1
    assert hs.hs_reuse_frame(0, 960 * 480, 28800, 0, 960, 27, 497) == -1


def test_spl_factor(hs, oracle):
    x = np.random.default_rng(4).uniform(-0.5, 0.5, 10000)
    y = 0.25 * x[:9000]
    er, ed = float(np.sum(x * x)), float(np.sum(y * y))
    f = hs.hs_spl_factor(er, x.size, ed, y.size)
    ref_spl = 20 * math.log10(math.sqrt(er / x.size) / 2e-5)
    deg_spl = 20 * math.log10(math.sqrt(ed / y.size) / 2e-5)
    assert f == oracle.zig_pow(10.0, (ref_spl - deg_spl) / 20.0)
    assert hs.hs_spl_factor(0.0, 10, ed, y.size) == 1.0


def test_svr(hs, oracle, kats):
    obs = np.array(kats["svr_default_known"]["obs"])
    y = c_double()
    assert hs.hs_svr_predict(None, 0, d(obs), ctypes.byref(y)) == 0
    assert y.value == oracle.svr_predict(obs)
    k = kats["svr_manual_rbf"]
    t = k["model"].encode()
    obs = np.array(k["obs"])
    assert hs.hs_svr_predict(t, len(t), d(obs), ctypes.byref(y)) == 0
    assert abs(y.value - k["expected"][0]) <= k["expected"][1]
    bad = b"svm_type c_svc\nSV\n1 1:1\n"
    assert hs.hs_svr_predict(bad, len(bad), d(obs), ctypes.byref(y)) == -4


def _wav(fmt, bits, nch, payload, rate=48000):
    hdr = b"RIFF" + struct.pack("<I", 36 + len(payload)) + b"WAVEfmt " + struct.pack(
        "<IHHIIHH", 16, fmt, nch, rate, rate * nch * bits // 8, nch * bits // 8, bits)
    return hdr + b"data" + struct.pack("<I", len(payload)) + payload


def test_decode_wav(hs):
    # reference src/audio.zig:178-199
    out, rate = np.zeros(16), c_uint32()
    w = _wav(1, 16, 2, bytes([0x00, 0x40, 0x00, 0xC0, 0xFF, 0x7F, 0xFF, 0x7F]))
    assert hs.hs_decode_wav(w, len(w), d(out), 16, ctypes.byref(rate)) == 2
    assert out[0] == 0.0 and out[1] == 32767.0 / 32768.0 and rate.value == 48000
    w = _wav(3, 32, 1, struct.pack("<ff", 0.5, -0.25))
    assert hs.hs_decode_wav(w, len(w), d(out), 16, ctypes.byref(rate)) == 2
    assert out[0] == 0.5 and out[1] == -0.25
    assert hs.hs_decode_wav(b"RIFX0000WAVE", 12, d(out), 16, ctypes.byref(rate)) == -3


def _bounds(hs, sizes, chunks, lanes, front):
    s = np.ascontiguousarray(sizes, dtype=np.uintp)
    out = np.zeros(len(s) + 1, dtype=np.uintp)
    k = hs.hs_chunk_bounds(s.ctypes.data_as(POINTER(c_size_t)), len(s), chunks, lanes, front,
                           out.ctypes.data_as(POINTER(c_size_t)))
    return out[:k].tolist()


def test_chunk_bounds_cases(hs):
    """The lanes' chunk queues (host and device inputs): consecutive pairs cut
    at cumulative size targets, the first `lanes` chunks at front% of the
    average."""
    assert _bounds(hs, [], 6, 2, 30) == [0]
    assert _bounds(hs, [7], 6, 2, 30) == [0, 1]
    assert _bounds(hs, [1] * 10, 5, 1, 0) == [0, 2, 4, 6, 8, 10]
    assert _bounds(hs, [1] * 10, 5, 1, 100) == [0, 2, 4, 6, 8, 10]
    # 100 equal pairs, 10 chunks over 5 lanes: average 10, the first five at 3,
    # the other five at (100 - 15) / 5 = 17
    assert _bounds(hs, [1] * 100, 10, 5, 30) == [0, 3, 6, 9, 12, 15, 32, 49, 66, 83, 100]
    # no more chunks than lanes: equal chunks whatever the front
    assert _bounds(hs, [1] * 12, 4, 4, 30) == [0, 3, 6, 9, 12]
    # a large pair first passes several targets but makes one chunk
    assert _bounds(hs, [100, 1, 1, 1], 4, 2, 0) == [0, 1, 2, 3, 4]
    # a large pair last: the small ones reach no target, one chunk
    assert _bounds(hs, [1, 1, 1, 100], 4, 1, 0) == [0, 4]
    assert _bounds(hs, [0, 0, 0], 3, 1, 30) == [0, 1, 2, 3]
    assert _bounds(hs, [5, 5], 8, 2, 30) == [0, 1, 2]


def test_chunk_bounds_properties(hs):
    rng = np.random.default_rng(5)
    for _ in range(300):
        n = int(rng.integers(1, 200))
        sizes = rng.integers(0, 1 << 24, n)
        if rng.random() < 0.2:
            sizes[rng.integers(n)] = 1 << 30
        lanes = int(rng.integers(1, 9))
        chunks = int(rng.integers(1, 4 * lanes + 1))
        front = int(rng.choice([0, 10, 30, 50, 99, 100, 150]))
        b = _bounds(hs, sizes, chunks, lanes, front)
        assert b[0] == 0 and b[-1] == n
        assert all(x < y for x, y in zip(b, b[1:])), b
        assert len(b) - 1 <= min(n, chunks)
        # the greedy rule: a chunk ends at the first pair whose running total
        # reaches that chunk's target, so no chunk ends early
        K = min(n, chunks)
        total = float(sizes.sum())
        if 0 < front < 100 and K > lanes:
            small = total / K * front / 100
            rest = (total - small * lanes) / (K - lanes)
            steps = [small if k < lanes else rest for k in range(K)]
        else:
            steps = [total / K] * K
        acc = np.cumsum(sizes)
        at = 0.0
        for k, e in enumerate(b[1:-1]):
            at += steps[k]
            assert acc[e - 1] >= int(at) - 1, (k, e)
            if e - 1 > b[k]:
                assert acc[e - 2] < int(at) + 1, (k, e)
