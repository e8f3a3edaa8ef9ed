"""Host-input batches whose uploads overlap scoring (chunks uploaded on a
copy stream while earlier chunks are scored: lanes sharing a queue of
chunks, or one lane chunking its own batch into two device slots) give
exactly the results of the same pairs uploaded all at once, and of the pairs
given as device inputs: every pair's result depends only on its own signals,
so chunking changes nothing but the timing. The byte bound below which
batches take the direct path is lowered here so that small batches split
into several chunks."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fields(res):
    keys = ("moslqo", "vnsim", "alignment_lag_s", "fvnsim", "fvnsim10", "fstdnsim", "fvdegenergy")
    return {k: np.asarray(res[k]) for k in keys}


def _same(a, b):
    (ca, ra, ta), (cb, rb, tb) = a, b
    assert ca == cb
    if ca != 0:
        return
    fa, fb = _fields(ra), _fields(rb)
    for k in fa:
        assert np.array_equal(fa[k], fb[k]), k
    for k in ("global_lag", "spl_factor", "nf_deg", "ref_index", "deg_offset", "realign_lag", "realign_accepted"):
        assert np.array_equal(np.asarray(ta[k]), np.asarray(tb[k])), k


def _device_run(ctx, refs, degs, sr):
    import torch
    d_ref = [torch.from_numpy(r).cuda() for r in refs]
    d_deg = [torch.from_numpy(d).cuda() for d in degs]
    torch.cuda.synchronize()
    return ctx.measure_batch_traced([t.data_ptr() for t in d_ref], [t.data_ptr() for t in d_deg], sr,
                                    device_inputs=True, ref_lens=[t.numel() for t in d_ref],
                                    deg_lens=[t.numel() for t in d_deg])


def _check(monkeypatch, ctx, refs, degs, sr):
    monkeypatch.setenv("VISQOL_STREAMED_MIN_BYTES", "1")
    monkeypatch.setenv("VISQOL_STREAMED_UPLOADS", "1")
    streamed = ctx.measure_batch_traced(refs, degs, sr)
    again = ctx.measure_batch_traced(refs, degs, sr)  # slots reused
    monkeypatch.setenv("VISQOL_STREAMED_UPLOADS", "0")
    direct = ctx.measure_batch_traced(refs, degs, sr)
    device = _device_run(ctx, refs, degs, sr)
    for s, a, d, v in zip(streamed, again, direct, device):
        _same(s, d)
        _same(a, d)
        _same(v, d)
    return streamed


@pytest.mark.parametrize("lanes", ["1", "4"])
@pytest.mark.parametrize("precision", ["exact", "fast"])
def test_streamed_audio_uneven(native, monkeypatch, precision, lanes):
    """One lane: the lane chunks its own batch (Engine::measure_batch_streamed);
    four lanes: the lanes share a queue of chunks uploaded in order."""
    from akvisqol_b200 import synth
    pairs = synth.audio_batch(9, seed0=synth.SEED_BASE + 300, min_s=2.0, max_s=7.0)
    refs, degs = [p[0] for p in pairs], [p[1] for p in pairs]
    # one pair too short to score: its error code comes back unchanged
    refs.insert(4, refs[4][:1000].copy())
    degs.insert(4, degs[4][:1000].copy())
    monkeypatch.setenv("VISQOL_GPU_LANES", lanes)
    ctx = native.Context(mode=native.MODE_AUDIO, precision=precision)
    got = _check(monkeypatch, ctx, refs, degs, 48000)
    assert got[4][0] != 0
    assert sum(1 for c, _, _ in got if c == 0) == len(refs) - 1


def test_streamed_speech_vad(native, monkeypatch):
    """Speech mode reads the host references for the VAD."""
    from akvisqol_b200 import synth
    pairs = synth.speech_batch(7, seed0=synth.SEED_BASE + 400, min_s=2.0, max_s=6.0)
    ctx = native.Context(mode=native.MODE_SPEECH, use_lattice_model=False, precision="exact")
    got = _check(monkeypatch, ctx, [p[0] for p in pairs], [p[1] for p in pairs], 16000)
    assert all(c == 0 for c, _, _ in got)


def test_streamed_prepared(native, monkeypatch):
    """Prepared references upload only the degraded signals."""
    from akvisqol_b200 import synth
    pairs = synth.audio_batch(6, seed0=synth.SEED_BASE + 500, min_s=2.0, max_s=5.0)
    refs, degs = [p[0] for p in pairs], [p[1] for p in pairs]
    ctx = native.Context(mode=native.MODE_AUDIO, precision="exact")
    prep = ctx.prepare(refs, 48000)

    def scores():
        out = []
        for o in ctx.measure_prepared(prep, degs):
            assert not isinstance(o, native.NativeError), o
            out.append(native.result_dict(o.contents))
            native.free(o)
        return out

    monkeypatch.setenv("VISQOL_STREAMED_MIN_BYTES", "1")
    monkeypatch.setenv("VISQOL_STREAMED_UPLOADS", "1")
    streamed = scores()
    monkeypatch.setenv("VISQOL_STREAMED_UPLOADS", "0")
    direct = scores()
    for s, d in zip(streamed, direct):
        assert s["moslqo"] == d["moslqo"]
        assert np.array_equal(s["fvnsim"], d["fvnsim"])


@pytest.mark.parametrize("precision", ["fast", "balanced"])
def test_device_inputs_chunk_queue(native, monkeypatch, precision):
    """Device-input batches of the FMA forms go through a queue of chunks
    (three a lane, the first round small) that the lanes take as they free
    up: the results are those of one share a lane and of host inputs, bit
    for bit, in the pairs' order."""
    from akvisqol_b200 import synth
    pairs = synth.audio_batch(8, seed0=synth.SEED_BASE + 600, min_s=2.0, max_s=6.0)
    refs, degs = [p[0] for p in pairs], [p[1] for p in pairs]
    monkeypatch.setenv("VISQOL_GPU_LANES", "2")
    ctx = native.Context(mode=native.MODE_AUDIO, precision=precision)
    monkeypatch.setenv("VISQOL_DEVICE_CHUNKS", "3")
    queued = _device_run(ctx, refs, degs, 48000)
    again = _device_run(ctx, refs, degs, 48000)
    monkeypatch.setenv("VISQOL_DEVICE_CHUNKS", "0")
    shares = _device_run(ctx, refs, degs, 48000)
    monkeypatch.setenv("VISQOL_STREAMED_UPLOADS", "0")
    host = ctx.measure_batch_traced(refs, degs, 48000)
    assert all(c == 0 for c, _, _ in queued)
    for q, a, s, h in zip(queued, again, shares, host):
        _same(q, s)
        _same(a, s)
        _same(h, s)
