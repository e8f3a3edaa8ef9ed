"""The request server (continuous batching): every request's result equals
the result of scoring the pair alone through a context, whatever else was in
flight with it; stats and admission limits behave as declared."""

import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mix(n_audio, n_speech):
    from akvisqol_b200 import synth
    reqs = [(0, p, 48000) for p in synth.audio_batch(n_audio, min_s=2.0, max_s=8.0)]
    reqs += [(1, p, 16000) for p in synth.speech_batch(n_speech, min_s=2.0, max_s=6.0)]
    order = np.random.default_rng(7).permutation(len(reqs))
    return [reqs[i] for i in order]


def _alone(native, precision, mode, pair, sr):
    ctx = native.Context(mode=mode, use_lattice_model=False, precision=precision)
    out = ctx.measure(pair[0], pair[1], sr)
    try:
        return native.result_dict(out.contents)
    finally:
        native.free(out)


@pytest.mark.parametrize("precision", ["exact", "fast"])
def test_results_same_alone_and_in_the_mix(native, precision):
    reqs = _mix(10, 6)
    server = native.Server(precision=precision, lanes=3, max_batch=4)
    tickets = {}

    def producer():
        rng = np.random.default_rng(11)
        for k, (mode, pair, sr) in enumerate(reqs):
            tickets[server.submit(mode, pair[0], pair[1], sr)] = k
            time.sleep(float(rng.exponential(0.004)))

    th = threading.Thread(target=producer)
    th.start()
    got = {}
    while len(got) < len(reqs):
        item = server.next(timeout_ms=60000)
        assert item is not None, "request did not complete"
        t, status, res = item
        assert status == 0
        got[t] = res
    th.join()
    st = server.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0 and st["queued"] == 0 and st["in_flight"] == 0
    assert 0 < st["latency_p50_ms"] <= st["latency_p99_ms"]
    assert st["batches"] >= 1 and st["mean_batch"] >= 1
    server.close()
    for t, res in got.items():
        mode, pair, sr = reqs[tickets[t]]
        want = _alone(native, precision, mode, pair, sr)
        assert res["moslqo"] == want["moslqo"]
        assert np.array_equal(res["fvnsim"], want["fvnsim"])
        assert np.array_equal(res["fstdnsim"], want["fstdnsim"])


def test_budget_rejects_oversize_pair(native):
    from akvisqol_b200 import synth
    server = native.Server(precision="exact", lanes=2, hbm_budget_bytes=64 << 20)
    ref, deg = synth.audio_pair(1, seconds=30.0)
    with pytest.raises(native.NativeError) as e:
        server.submit(0, ref, deg, 48000)
    assert e.value.code == native.E_OUT_OF_MEMORY
    # a short pair fits and scores
    ref, deg = synth.audio_pair(2, seconds=2.0)
    server.submit(0, ref, deg, 48000)
    t, status, res = server.next(timeout_ms=60000)
    assert status == 0 and 1.0 <= res["moslqo"] <= 5.0
    server.close()


def test_failed_pair_is_isolated(native):
    from akvisqol_b200 import synth
    server = native.Server(precision="exact", lanes=1, max_batch=8)
    good = synth.audio_pair(3, seconds=3.0)
    bad = (np.zeros(100), np.zeros(100))  # shorter than one analysis window
    tg = server.submit(0, good[0], good[1], 48000)
    tb = server.submit(0, bad[0], bad[1], 48000)
    seen = {}
    for _ in range(2):
        t, status, res = server.next(timeout_ms=60000)
        seen[t] = (status, res)
    assert seen[tg][0] == 0 and seen[tg][1] is not None
    assert seen[tb][0] != 0 and seen[tb][1] is None
    st = server.stats()
    assert st["completed"] == 1 and st["failed"] == 1
    server.close()


def test_pending_when_idle(native):
    server = native.Server(precision="exact", lanes=1)
    assert server.next(timeout_ms=10) is None
    server.close()


def test_pooled_budget_admits_pair_larger_than_a_lane_share(native):
    """HBM is one pool: with four lanes and a budget of 1.5 footprints, a pair
    of one footprint (more than a quarter of the budget) is admitted, each in
    turn, and scores as it does alone; a pair larger than the whole budget is
    refused."""
    from akvisqol_b200 import synth
    pairs = [synth.audio_pair(synth.SEED_BASE + 60 + i, seconds=6.0) for i in range(3)]
    foot = max(native.pair_footprint(r.size, d.size, 48000) for r, d in pairs)
    server = native.Server(precision="exact", lanes=4, max_batch=8, hbm_budget_bytes=foot * 3 // 2)
    tickets = {server.submit(0, r, d, 48000): k for k, (r, d) in enumerate(pairs)}
    got = {}
    for _ in pairs:
        t, status, res = server.next(timeout_ms=120000)
        assert status == 0
        got[tickets[t]] = res
    st = server.stats()
    assert st["completed"] == 3 and st["failed"] == 0 and st["mean_batch"] == 1.0
    big = synth.audio_pair(synth.SEED_BASE + 70, seconds=12.0)
    assert native.pair_footprint(big[0].size, big[1].size, 48000) > foot * 3 // 2
    with pytest.raises(native.NativeError) as e:
        server.submit(0, big[0], big[1], 48000)
    assert e.value.code == native.E_OUT_OF_MEMORY
    server.close()
    for k, (r, d) in enumerate(pairs):
        want = _alone(native, "exact", 0, (r, d), 48000)
        assert got[k]["moslqo"] == want["moslqo"]
