"""The reference's own, unchanged Python package scoring through this
library on the GPU: the drop-in boundary seen from the caller's side.

The package (reference src/python/visqol: visqol_lib_py.VisqolApi,
src/python/visqol/visqol_lib_py.py:221-226, and _native.Context,
src/python/visqol/_native.py:165-234) loads libvisqol through ctypes from
VISQOL_LIBRARY and picks its backend from VISQOL_BACKEND; here both point
at this build (backend cuda). It runs in a fresh interpreter, and its MOS
and per-band features are compared with the oracle at 1e-12.

The package is not part of this repository: VISQOL_REFERENCE_PYTHON names
the reference's src/python directory (its src/model beside it holds the
default models). Without it the test is skipped.
"""

import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

REF_PY = os.environ.get("VISQOL_REFERENCE_PYTHON")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not REF_PY or not Path(REF_PY, "visqol", "_native.py").is_file(),
                                 reason="VISQOL_REFERENCE_PYTHON does not name the reference's src/python")]

SCRIPT = r"""
import json, sys
import numpy as np
from visqol import _native, visqol_lib_py
from visqol.pb2 import visqol_config_pb2

d = np.load(sys.argv[1])
out = {"abi": int(_native.lib.visqol_abi_version()), "backends": _native.available_backends()}

def api(speech, rate, ref, deg):
    cfg = visqol_config_pb2.VisqolConfig()
    cfg.audio.sample_rate = rate
    cfg.options.use_speech_scoring = speech
    cfg.options.use_lattice_model = False
    cfg.options.search_window_radius = 60
    a = visqol_lib_py.VisqolApi()
    a.Create(cfg)
    m = a.Measure(ref, deg)
    return {"moslqo": m.moslqo, "vnsim": m.vnsim, "fvnsim": list(m.fvnsim), "fstdnsim": list(m.fstdnsim),
            "alignment_lag_s": m.alignment_lag_s}

out["audio"] = api(False, 48000, d["ar"], d["ad"])
out["speech"] = api(True, 16000, d["sr"], d["sd"])

ctx = _native.Context(mode=_native.MODE_AUDIO, search_window_radius=60, use_unscaled_speech_mos_mapping=False,
                      disable_global_alignment=False, disable_realignment=False, use_lattice_model=False,
                      model_path=None, backend="cuda", precision="exact")
got = ctx.measure_batch([d["ar"], d["br"]], [d["ad"], d["bd"]], 48000, 0)
out["batch"] = []
for r in got:
    out["batch"].append({"moslqo": r.contents.moslqo, "fvnsim": _native.vec(r.contents.fvnsim, 32).tolist()})
    _native.free(r)
print(json.dumps(out))
"""


def test_reference_package_scores_on_this_library(native, oracle, tmp_path):
    from akvisqol_b200 import synth
    ar, ad = synth.audio_pair(synth.SEED_BASE)  # 10 s 48 kHz audio
    br, bd = synth.audio_pair(synth.SEED_BASE + 1, seconds=4.0)
    sr, sd = synth.speech_pair(synth.SEED_BASE)  # 8 s 16 kHz speech
    np.savez(tmp_path / "pairs.npz", ar=ar, ad=ad, br=br, bd=bd, sr=sr, sd=sd)
    env = dict(os.environ, PYTHONPATH=REF_PY, VISQOL_LIBRARY=str(native.LIB_PATH), VISQOL_BACKEND="cuda")
    p = subprocess.run([sys.executable, "-c", SCRIPT, str(tmp_path / "pairs.npz")], env=env, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-3000:]
    got = json.loads(p.stdout.strip().splitlines()[-1])
    assert got["abi"] == 1 and "cuda" in got["backends"]

    want, _ = oracle.measure(ar, ad, 48000)
    assert abs(got["audio"]["moslqo"] - want["moslqo"]) <= 1e-12
    assert np.max(np.abs(np.array(got["audio"]["fvnsim"]) - want["fvnsim"])) <= 1e-12
    assert got["audio"]["alignment_lag_s"] == want["alignment_lag_s"]

    swant, _ = oracle.measure(sr, sd, 16000, oracle.options(mode=1))
    assert abs(got["speech"]["moslqo"] - swant["moslqo"]) <= 1e-12
    assert np.max(np.abs(np.array(got["speech"]["fvnsim"]) - swant["fvnsim"])) <= 1e-12

    bwant, _ = oracle.measure(br, bd, 48000)
    assert abs(got["batch"][0]["moslqo"] - want["moslqo"]) <= 1e-12
    assert abs(got["batch"][1]["moslqo"] - bwant["moslqo"]) <= 1e-12
