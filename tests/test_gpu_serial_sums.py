"""The exact form's serial statistics (visqol_b200_signal_sums) against the
CPU's left-to-right f64 sums, bit for bit (reference src/envelope.zig:28-41,
src/audio.zig:132-136). The kernels add whole tiles at once by an integer
form of the serial additions, valid while the running sum keeps its binade
and no addition is a rounding tie; these inputs cross binades, make ties,
start with silence, run negative, span the exponent range and carry inf and
NaN, so that both the shortcut and its fallback decide results."""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def serial(terms):
    s = 0.0
    for t in terms:
        s += t
    return s


def cpu_sums(x, skip):
    n = len(x)
    total = serial(x)
    nyq = 0.0
    if n:
        mean = total / n
        sign = 1.0
        for v in x:
            nyq += sign * (v - mean)
            sign = -sign
    sq = [v * v for v in x]
    first = next((k for k, v in enumerate(sq) if v != 0.0), n)
    return {"sum": total, "nyquist": nyq, "energy": serial(sq), "first_nonzero": first,
            "aligned_energy": serial(sq[skip:])}


def same(a, b):
    if isinstance(a, int):
        return a == b
    if math.isnan(a) or math.isnan(b):
        return math.isnan(a) and math.isnan(b)
    return np.float64(a).view(np.int64) == np.float64(b).view(np.int64)


def check(native, x, skip=0):
    x = np.ascontiguousarray(x, dtype=np.float64)
    got = native.signal_sums(x, skip)
    want = cpu_sums(x.tolist(), skip)
    for key, v in want.items():
        assert same(got[key], v), (key, got[key], v, len(x))


def cases():
    rng = np.random.default_rng(71)
    out = {}
    out["gauss"] = rng.standard_normal(480000) * 0.1
    pcm = np.round(rng.standard_normal(100000) * 3000) / 32768.0
    out["pcm_after_silence"] = np.concatenate([np.zeros(1776), pcm])
    out["negative_dc"] = -0.3 + 0.01 * rng.standard_normal(70001)
    # ties: 1 + 2^-53 rounds to even, so the sum sits still or steps by two units
    out["ties_even"] = np.array([1.0] + [2.0 ** -53] * 3000)
    out["ties_odd"] = np.array([1.0 + 2.0 ** -52] + [2.0 ** -53] * 3000)
    out["ties_mixed"] = np.where(rng.random(5000) < 0.5, 2.0 ** -53, 3 * 2.0 ** -53)
    out["ties_mixed"][0] = 1.0
    # sums that land exactly on powers of two
    out["binade_edges"] = np.full(5000, 0.25)
    mags = 10.0 ** rng.uniform(-300, 300, 20000)
    out["exponent_range"] = mags * np.where(rng.random(20000) < 0.5, -1.0, 1.0)
    out["subnormals"] = np.array([5e-324, 1e-310, -5e-324, 2.5e-308] * 300)
    walk = rng.standard_normal(60000)
    walk[::997] *= 1e6
    out["wandering"] = walk
    out["zeros"] = np.zeros(3000)
    out["negative_zeros"] = -np.zeros(700)
    out["inf"] = np.array([1.0, np.inf, 2.0] * 100)
    out["nan"] = np.concatenate([rng.standard_normal(600), [np.inf, -np.inf], rng.standard_normal(600)])
    for n in (1, 7, 255, 256, 257, 2047, 65539):
        out[f"len{n}"] = rng.standard_normal(n) * 0.05
    return out


CASES = cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_serial_sums_bit_exact(native, name):
    check(native, CASES[name])


@pytest.mark.parametrize("skip", [0, 1, 255, 1777, 4000])
def test_aligned_energy_windows(native, skip):
    rng = np.random.default_rng(skip)
    x = np.concatenate([np.zeros(1776), rng.standard_normal(3000) * 0.2])
    check(native, x, skip=min(skip, len(x)))


def test_empty_signal(native):
    got = native.signal_sums(np.zeros(0))
    assert got["sum"] == 0.0 and got["nyquist"] == 0.0 and got["energy"] == 0.0
    assert got["first_nonzero"] == 0 and got["aligned_energy"] == 0.0


@pytest.mark.parametrize("kind", ["audio", "speech"])
def test_bench_signals(native, kind):
    from akvisqol_b200 import synth
    if kind == "audio":
        ref, deg = synth.audio_pair(synth.SEED_BASE, seconds=10.0)
    else:
        ref, deg = synth.speech_pair(synth.SEED_BASE + 0x8000, seconds=8.0)
    check(native, ref, skip=1778)
    check(native, deg, skip=1778)
