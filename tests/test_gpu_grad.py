"""d moslqo / d degraded signal (visqol_b200_measure_batch_grad) against
central differences of the oracle's score, as the reference checks its
gradient (README.md:215-236, src/gpu/pipeline.zig:842-1143): the forward
pass's discrete choices (lags, matches, realignment, selected floor and
minimum cells) held fixed, a small step changes none of them."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

H = 1e-4


def central(oracle, ref, deg, sr, opts, k):
    dp, dm = deg.copy(), deg.copy()
    dp[k] += H
    dm[k] -= H
    up = oracle.measure(ref, dp, sr, opts, trace=False)[0]["moslqo"]
    dn = oracle.measure(ref, dm, sr, opts, trace=False)[0]["moslqo"]
    return (up - dn) / (2 * H)


def check(native, oracle, ref, deg, sr, mode, precision, opts, picks=10, seed=0):
    ctx = native.Context(mode=mode, use_lattice_model=False, precision=precision)
    (code, res, grad), = ctx.measure_batch_grad([ref], [deg], sr)
    assert code == 0 and grad.shape == deg.shape and np.all(np.isfinite(grad))
    want = oracle.measure(ref, deg, sr, opts, trace=False)[0]["moslqo"]
    assert abs(res["moslqo"] - want) <= (1e-12 if precision == "exact" else 1e-6)
    rng = np.random.default_rng(seed)
    top = np.argsort(-np.abs(grad))[:picks]
    rand = rng.choice(deg.size, picks, replace=False)
    worst = 0.0
    for k in np.concatenate([top, rand]):
        fd = central(oracle, ref, deg, sr, opts, int(k))
        err = abs(grad[k] - fd)
        assert err <= 1e-3 * abs(fd) + 1e-8, (int(k), grad[k], fd)
        worst = max(worst, err / max(abs(fd), 1e-8))
    return grad


@pytest.mark.parametrize("precision", ["exact", "balanced", "fast"])
def test_audio_gradient(native, oracle, precision):
    from akvisqol_b200 import synth
    ref, deg = synth.audio_pair(synth.SEED_BASE + 3, seconds=3.0)
    grad = check(native, oracle, ref, deg, 48000, native.MODE_AUDIO, precision, oracle.options())
    # the prepended delay's samples are dropped by the lag: no gradient
    assert np.all(grad[:1700] == 0.0)


def test_speech_gradient(native, oracle):
    from akvisqol_b200 import synth
    ref, deg = synth.speech_pair(synth.SEED_BASE + 4, seconds=3.0)
    check(native, oracle, ref, deg, 16000, native.MODE_SPEECH, "exact", oracle.options(mode=1))


def test_gradient_through_realigned_slices(native, oracle):
    """A pair whose degraded signal gains 7 samples of delay half way: the
    first half's patches realign off the frame grid, so their statistics
    come from recomputed slice spectrograms whose reverse runs on its own."""
    from akvisqol_b200 import synth
    ref, deg = synth.audio_pair(synth.SEED_BASE + 5, seconds=4.0)
    k = len(deg) // 2
    deg = np.concatenate([deg[:k], np.zeros(7), deg[k:]])
    tr = oracle.measure(ref, deg, 48000)[1]
    assert np.any(tr["realign_accepted"] & (tr["realign_lag"] != 0))
    check(native, oracle, ref, deg, 48000, native.MODE_AUDIO, "exact", oracle.options(), seed=1)
