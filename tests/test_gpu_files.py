"""The WAV-file entry points through the C ABI (reference visqol_measure_files
and visqol_measure_files_batch, src/capi.zig:300-456; WAV decoding
src/audio.zig:41-112): files the test writes in several encodings, scored on
the GPU and checked against the oracle on the same decoded samples."""

import struct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def write_wav(path, x, rate, kind, channels=1):
    """x (frames,) or (frames, channels) in [-1, 1) as a RIFF/WAVE file;
    returns the samples a decoder gives back, mono-averaged."""
    x = np.asarray(x, np.float64)
    if x.ndim == 1:
        x = np.repeat(x[:, None], channels, axis=1)
    if kind == "pcm16":
        q = np.clip(np.round(x * 32768.0), -32768, 32767).astype("<i2")
        tag, bits, data, back = 1, 16, q.tobytes(), q.astype(np.float64) / 32768.0
    elif kind == "pcm24":
        q = np.clip(np.round(x * 8388608.0), -8388608, 8388607).astype(np.int64)
        u = (q & 0xFFFFFF).astype("<u4")
        data = np.stack([(u >> s & 0xFF).astype(np.uint8) for s in (0, 8, 16)], axis=-1).tobytes()
        tag, bits, back = 1, 24, q.astype(np.float64) / 8388608.0
    elif kind == "float32":
        f = x.astype("<f4")
        tag, bits, data, back = 3, 32, f.tobytes(), f.astype(np.float64)
    else:
        raise ValueError(kind)
    ch = x.shape[1]
    block = ch * bits // 8
    fmt = struct.pack("<HHIIHH", tag, ch, rate, rate * block, block, bits)
    body = b"WAVE" + b"fmt " + struct.pack("<I", len(fmt)) + fmt + b"data" + struct.pack("<I", len(data)) + data
    path.write_bytes(b"RIFF" + struct.pack("<I", len(body)) + body)
    return back[:, 0] if ch == 1 else back.sum(axis=1) / ch


def pair(seed, rate, seconds=3.0):
    from akvisqol_b200 import synth
    if rate == 48000:
        return synth.audio_pair(seed, seconds=seconds, sample_rate=rate)
    return synth.audio_pair(seed, seconds=seconds, sample_rate=rate, cutoff_hz=0.4 * rate)


def test_measure_files_matches_oracle(native, oracle, tmp_path):
    ref, deg = pair(0x5EED_7000, 48000)
    r = write_wav(tmp_path / "r.wav", ref, 48000, "pcm16")
    d = write_wav(tmp_path / "d.wav", deg, 48000, "pcm24")
    ctx = native.Context(mode=native.MODE_AUDIO, precision="exact")
    out = ctx.measure_files(str(tmp_path / "r.wav"), str(tmp_path / "d.wav"))
    try:
        got = out.contents.moslqo
    finally:
        native.free(out)
    want, _ = oracle.measure(r, d, 48000)
    assert abs(got - want["moslqo"]) <= 1e-12


def test_measure_files_batch_mixed_rates_and_failures(native, oracle, tmp_path):
    """One batch: 48 and 16 kHz pairs (grouped by rate inside the call), 16-bit,
    24-bit, float and stereo encodings, a missing file (that pair alone
    fails with VISQOL_E_IO and a NULL result) and a pair whose two files
    differ in rate (VISQOL_E_SIGNAL)."""
    specs = [(48000, "pcm16", 1), (16000, "pcm24", 1), (48000, "float32", 1), (16000, "pcm16", 2),
             (48000, "pcm24", 2)]
    refs, degs, want = [], [], []
    for k, (rate, kind, ch) in enumerate(specs):
        ref, deg = pair(0x5EED_7100 + k, rate)
        rp, dp = tmp_path / f"r{k}.wav", tmp_path / f"d{k}.wav"
        r = write_wav(rp, ref, rate, kind, ch)
        d = write_wav(dp, deg, rate, kind, ch)
        refs.append(str(rp))
        degs.append(str(dp))
        want.append(oracle.measure(r, d, rate)[0]["moslqo"])
    refs.append(str(tmp_path / "missing.wav"))
    degs.append(degs[0])
    ref, deg = pair(0x5EED_7200, 48000)
    write_wav(tmp_path / "r48.wav", ref, 48000, "pcm16")
    write_wav(tmp_path / "d16.wav", deg[::3], 16000, "pcm16")
    refs.append(str(tmp_path / "r48.wav"))
    degs.append(str(tmp_path / "d16.wav"))

    ctx = native.Context(mode=native.MODE_AUDIO, precision="exact")
    got = ctx.measure_files_batch(refs, degs)
    assert len(got) == len(specs) + 2
    for k in range(len(specs)):
        assert not isinstance(got[k], native.NativeError), got[k]
        try:
            assert abs(got[k].contents.moslqo - want[k]) <= 1e-12, (specs[k], got[k].contents.moslqo, want[k])
        finally:
            native.free(got[k])
    assert isinstance(got[-2], native.NativeError) and got[-2].code == native.E_IO
    assert isinstance(got[-1], native.NativeError) and got[-1].code == native.E_SIGNAL
