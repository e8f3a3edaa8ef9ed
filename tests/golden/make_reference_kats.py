"""Extract the reference's self-contained known-answer vectors into
reference_kats.json.

The reference (jdek/akvisqol, Zig) cannot be built in this image, so its own
unit tests are read as text: each named `test "..." { ... }` block below is
located in the reference source and its literal arrays and expected values
are copied out. Run from the repository root with the reference checked out:

    python tests/golden/make_reference_kats.py /path/to/akvisqol

The JSON it writes is committed; tests read only the JSON.
"""

import json
import re
import sys
from pathlib import Path

NUM = r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?"


def test_body(src: str, name: str) -> str:
    start = src.index(f'test "{name}"')
    brace = src.index("{", start)
    depth = 0
    for i in range(brace, len(src)):
        if src[i] == "{":
            depth += 1
        elif src[i] == "}":
            depth -= 1
            if depth == 0:
                return src[brace + 1:i]
    raise ValueError(name)


def literal(body: str, var: str):
    """Numbers of `const/var <var> ... = ...{ ... };` (nested braces flattened, row order kept)."""
    m = re.search(r"(?:const|var)\s+" + re.escape(var) + r"\b[^=]*=\s*", body)
    if not m:
        raise ValueError(var)
    i = body.index("{", m.end())
    depth = 0
    for j in range(i, len(body)):
        if body[j] == "{":
            depth += 1
        elif body[j] == "}":
            depth -= 1
            if depth == 0:
                text = body[i:j + 1]
                break
    rows = []
    # 2-D literals: one list per inner brace group.
    inner = re.findall(r"\{([^{}]*)\}", text)
    for grp in inner:
        rows.append([float(x) for x in re.findall(NUM, grp)])
    return rows if len(rows) > 1 else rows[0]


def approx(body: str):
    """(expected, tolerance) of every expectApproxEqAbs(@as(f64, E), _, T)."""
    consts = {m.group(1): float(m.group(2)) for m in re.finditer(r"const\s+(\w+)\s*=\s*(" + NUM + r")\s*;", body)}
    out = []
    for m in re.finditer(r"expectApproxEqAbs\(@as\(f64,\s*(" + NUM + r")\),\s*[^,]+,\s*(\w[\w.+-]*)\)", body):
        tol = m.group(2)
        out.append([float(m.group(1)), consts[tol] if tol in consts else float(tol)])
    return out


def main(ref_root: Path, out: Path) -> None:
    src = {p: (ref_root / "src" / p).read_text() for p in [
        "dsp/erb.zig", "gammatone.zig", "spectrogram.zig", "envelope.zig", "xcorr.zig",
        "nsim.zig", "dp.zig", "realign.zig", "vad.zig", "audio.zig", "svr.zig"]}
    k = {"source": "jdek/akvisqol src/*.zig inline tests, extracted by make_reference_kats.py"}

    b = test_body(src["dsp/erb.zig"], "uniformCenterFreqs first/last match reference")
    k["erb_center_freqs"] = {"n": 32, "low": 50.0, "high": 24000.0, "first_last": approx(b),
                             "cite": "src/dsp/erb.zig:64-72"}

    b = test_body(src["gammatone.zig"], "Filters: lowest band reference output (first 3 samples)")
    k["gammatone_lowest_band"] = {"samples": literal(b, "samples"), "expected": approx(b),
                                  "cite": "src/gammatone.zig:491-505"}
    b = test_body(src["gammatone.zig"], "Filters: 32-band 48kHz center freqs are sorted ascending")
    k["gammatone_center_freqs"] = {"first_last": approx(b), "cite": "src/gammatone.zig:469-478"}

    b = test_body(src["spectrogram.zig"], "convertToDbAndRaiseFloor: reference values")
    k["db_reference"] = {"data": literal(b, "data"), "expected": literal(b, "expected"), "tol": 1e-3,
                         "floor": -1000.0, "cite": "src/spectrogram.zig:95-103"}
    b = test_body(src["spectrogram.zig"], "convertToDbAndRaiseFloor: clamps to floor")
    k["db_clamp"] = {"data": literal(b, "data"), "expected": [e for e, _ in approx(b)], "floor": -45.0,
                     "cite": "src/spectrogram.zig:105-111"}
    b = test_body(src["spectrogram.zig"], "subtractJointMinimum: shifts both by the joint min")
    k["joint_min"] = {"a": literal(b, "a"), "b": literal(b, "b"), "expected": [e for e, _ in approx(b)],
                      "cite": "src/spectrogram.zig:113-123"}
    b = test_body(src["spectrogram.zig"], "raiseFloorPerFrame: clamps below per-column max minus threshold")
    k["floor_per_frame"] = {"ref": literal(b, "ref"), "deg": literal(b, "deg"),
                            "expected": [e for e, _ in approx(b)], "cite": "src/spectrogram.zig:125-138"}

    xc = src["xcorr.zig"]
    cases = []
    for name, want in [("bestLag: equal-length signals, positive lag of 2", 2),
                       ("bestLag: reference shorter than degraded → still 2", 2),
                       ("bestLag: reference longer than degraded → still 2", 2),
                       ("bestLag: negative lag of -2", -2),
                       ("bestLag: identical signals → lag 0", 0)]:
        b = test_body(xc, name)
        if "const sig" in b:
            s = literal(b, "sig")
            cases.append({"name": name, "ref": s, "deg": s, "lag": want})
        else:
            cases.append({"name": name, "ref": literal(b, "ref"), "deg": literal(b, "deg"), "lag": want})
    k["best_lag"] = {"cases": cases, "cite": "src/xcorr.zig:349-381"}
    b = test_body(xc, "fftSizeFor: next power of two of 2*biggest - 1")
    k["fft_size_for"] = {"pairs": [[int(m.group(2)), int(m.group(1))] for m in re.finditer(
        r"expectEqual\(@as\(usize, (\d+)\), fftSizeFor\((\d+)\)\)", b)], "cite": "src/xcorr.zig:342-347"}

    b = test_body(src["nsim.zig"], "conv2d3x3Replicate: reference output")
    k["conv2d"] = {"cols": literal(b, "cols"), "expected_cols": literal(b, "exp_cols"), "tol": 1e-3,
                   "cite": "src/nsim.zig:513-548"}
    b = test_body(src["nsim.zig"], "Comparator.measurePatchSimilarity: reference test_neurogram_measure")
    k["patch_similarity_3x1"] = {"ref": literal(b, "ref"), "deg": literal(b, "deg"),
                                 "expected_means": [e for e, _ in approx(b)], "tol": 1e-4,
                                 "cite": "src/nsim.zig:550-568"}

    d = src["dp.zig"]
    b = test_body(d, "refPatchIndices: sliding indices")
    k["ref_patch_indices"] = {"num_frames": 200, "patch": 30, "expected": [int(x) for x in literal(b, "expected")],
                              "cite": "src/dp.zig:389-396"}
    b = test_body(d, "calcMaxNumPatches: drops tail patches that exceed deg")
    k["calc_max_num_patches"] = {"idx": [int(x) for x in literal(b, "idx")],
                                 "cases": [[int(m.group(2)), int(m.group(3)), int(m.group(1))] for m in re.finditer(
                                     r"expectEqual\(@as\(usize, (\d+)\), calcMaxNumPatches\(&idx, (\d+), (\d+)\)\)", b)],
                                 "cite": "src/dp.zig:398-402"}
    b = test_body(d, "DP: optimal patch start times")
    k["dp_start_times"] = {"ref_rows": literal(b, "ref_rows"), "deg": literal(b, "deg_col_major"),
                           "num_bands": 3, "nf_ref": 10, "nf_deg": 30, "patch": 1, "radius": 8,
                           "frame_duration": 1.0, "indices": list(range(10)),
                           "expected": {str(m.group(2)): float(m.group(1)) for m in re.finditer(
                               r"expectApproxEqAbs\(@as\(f64, (" + NUM + r")\), matches\.items\[(\d+)\]", b)},
                           "cite": "src/dp.zig:404-450"}

    b = test_body(src["realign.zig"], "sliceAudio: in-range slice copies samples")
    k["slice_in_range"] = {"signal": literal(b, "sig"), "sr": 10, "t0": 0.2, "t1": 0.6, "len": 4,
                           "first": 0.3, "last": 0.6, "cite": "src/realign.zig:462-470"}
    k["slice_padded"] = {"len": 48000, "one_at": 16000, "sr": 16000, "t0": 0.5, "t1": 2.5, "out_len": 32000,
                         "one_out_at": 8000, "cite": "src/realign.zig:472-482"}
    k["lag_samples_back"] = {"lag": 27, "sr": 48000, "expected": 26, "cite": "src/realign.zig:528"}

    b = test_body(src["vad.zig"], "refPatchIndices: silence after the forced-active lead-in drops patches")
    k["vad"] = {"len": 64000, "active": [16000, 32000], "freq_per_sample": 0.1, "patch": 20, "window": 1280,
                "overlap": 0.25, "first": 9, "cite": "src/vad.zig:83-95"}

    b = test_body(src["audio.zig"], "soundPressureLevel: unit dc has known SPL")
    k["spl_unit_dc"] = {"n": 16, "expected": approx(b)[0], "cite": "src/audio.zig:201-204"}

    s = src["svr.zig"]
    b = test_body(s, "predict: matches manual RBF computation")
    txt = "".join(re.findall(r'"((?:[^"\\]|\\.)*)"', b.split("var m")[0])).encode().decode("unicode_escape")
    k["svr_manual_rbf"] = {"model": txt, "obs": literal(b, "obs"), "expected": approx(b)[0],
                           "cite": "src/svr.zig:190-201"}
    b = test_body(s, "predict: default SVR known FVNSIM observation → 4.30533")
    k["svr_default_known"] = {"obs": literal(b, "obs"), "expected": approx(b)[0], "cite": "src/svr.zig:203-219"}

    out.write_text(json.dumps(k, indent=1) + "\n")
    print(f"wrote {out} ({len(k) - 1} vectors)")


if __name__ == "__main__":
    import os
    where = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("VISQOL_REFERENCE_ROOT")
    if not where:
        sys.exit("usage: make_reference_kats.py <reference checkout> (or set VISQOL_REFERENCE_ROOT)")
    main(Path(where), Path(__file__).with_name("reference_kats.json"))
