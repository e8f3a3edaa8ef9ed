"""Prepared references: scoring against references prepared once gives the
same results as scoring the pairs directly, for every form and both modes."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert a["moslqo"] == b["moslqo"]
    for key in ("fvnsim", "fvnsim10", "fstdnsim", "fvdegenergy"):
        assert np.array_equal(a[key], b[key]), key
    assert len(a["patch_sims"]) == len(b["patch_sims"])
    for x, y in zip(a["patch_sims"], b["patch_sims"]):
        assert x["similarity"] == y["similarity"] and x["deg_patch_start_time"] == y["deg_patch_start_time"]


def _dicts(native, outs):
    res = []
    for o in outs:
        assert not isinstance(o, native.NativeError), o
        res.append(native.result_dict(o.contents))
        native.free(o)
    return res


@pytest.mark.parametrize("precision", ["exact", "balanced", "fast"])
@pytest.mark.parametrize("mode", [0, 1])
def test_prepared_equals_direct(native, precision, mode):
    from akvisqol_b200 import synth
    if mode == 0:
        pairs, sr = synth.audio_batch(6, min_s=3.0, max_s=6.0), 48000
    else:
        pairs, sr = synth.speech_batch(6, min_s=2.0, max_s=5.0), 16000
    refs = [p[0] for p in pairs[:3]]
    # two degraded signals per reference: its own and the next pair's
    ref_index = [0, 1, 2, 0, 1, 2]
    degs = [pairs[i][1] for i in range(6)]
    ctx = native.Context(mode=mode, use_lattice_model=False, precision=precision)
    prep = ctx.prepare(refs, sr)
    got = _dicts(native, ctx.measure_prepared(prep, degs, ref_index=ref_index))
    want = _dicts(native, ctx.measure_batch([refs[k] for k in ref_index], degs, sr))
    for g, w in zip(got, want):
        _same(g, w)


def test_prepared_device_inputs_and_reuse(native):
    import torch
    from akvisqol_b200 import synth
    pairs = synth.audio_batch(4, min_s=3.0, max_s=5.0)
    d_ref = [torch.from_numpy(p[0]).cuda() for p in pairs]
    d_deg = [torch.from_numpy(p[1]).cuda() for p in pairs]
    torch.cuda.synchronize()
    ctx = native.Context(mode=0, precision="exact")
    prep = ctx.prepare([t.data_ptr() for t in d_ref], 48000, device_inputs=True, ref_lens=[t.numel() for t in d_ref])
    want = _dicts(native, ctx.measure_batch([p[0] for p in pairs], [p[1] for p in pairs], 48000))
    for _ in range(2):  # the prepared references are read, never modified
        got = _dicts(native, ctx.measure_prepared(prep, [t.data_ptr() for t in d_deg], device_inputs=True,
                                                  deg_lens=[t.numel() for t in d_deg]))
        for g, w in zip(got, want):
            _same(g, w)


def test_prepared_errors(native):
    from akvisqol_b200 import synth
    ref, deg = synth.audio_pair(5, seconds=3.0)
    ctx = native.Context(mode=0, precision="exact")
    prep = ctx.prepare([ref, np.zeros(100)], 48000)
    outs = ctx.measure_prepared(prep, [deg, deg], ref_index=[0, 1])
    assert not isinstance(outs[0], native.NativeError)
    native.free(outs[0])
    assert isinstance(outs[1], native.NativeError) and outs[1].code == native.E_SIGNAL
    other = native.Context(mode=0, precision="fast")
    with pytest.raises(native.NativeError) as e:
        other.measure_prepared(prep, [deg])
    assert e.value.code == native.E_INVALID_ARGUMENT
    with pytest.raises(native.NativeError) as e:
        ctx.measure_prepared(prep, [deg], ref_index=[2])
    assert e.value.code == native.E_INVALID_ARGUMENT
