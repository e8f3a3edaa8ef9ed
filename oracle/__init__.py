"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is the checker: tests, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` import this module. The product library never
does.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_size_t, c_uint8, c_uint32, c_uint64
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "build" / "libvisqol_oracle.so"


def build() -> Path:
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


class Options(ctypes.Structure):
    _fields_ = [
        ("mode", c_uint32), ("search_window_radius", c_int32),
        ("use_unscaled_speech_mos_mapping", c_uint8), ("disable_global_alignment", c_uint8),
        ("disable_realignment", c_uint8), ("use_lattice_model", c_uint8),
        ("model_path", c_char_p), ("backend", c_uint32), ("precision", c_uint32),
    ]


class Patch(ctypes.Structure):
    _fields_ = [
        ("similarity", c_double), ("ref_patch_start_time", c_double), ("ref_patch_end_time", c_double),
        ("deg_patch_start_time", c_double), ("deg_patch_end_time", c_double),
        ("freq_band_means", POINTER(c_double)), ("freq_band_stddevs", POINTER(c_double)),
        ("freq_band_deg_energy", POINTER(c_double)),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("moslqo", c_double), ("vnsim", c_double), ("alignment_lag_s", c_double), ("num_bands", c_size_t),
        ("fvnsim", POINTER(c_double)), ("fvnsim10", POINTER(c_double)), ("fstdnsim", POINTER(c_double)),
        ("fvdegenergy", POINTER(c_double)), ("center_freq_bands", POINTER(c_double)),
        ("num_patches", c_size_t), ("patch_sims", POINTER(Patch)),
    ]


class Trace(ctypes.Structure):
    _fields_ = [
        ("global_lag", c_int64), ("spl_factor", c_double), ("deg_len", c_uint64),
        ("nf_ref", c_uint64), ("nf_deg", c_uint64), ("num_patches", c_uint64),
        ("ref_index", POINTER(c_int64)), ("deg_offset", POINTER(c_int64)), ("valid", POINTER(c_uint8)),
        ("realign_lag", POINTER(c_int64)), ("realign_frames", POINTER(c_int64)),
        ("realign_reused", POINTER(c_uint8)), ("realign_accepted", POINTER(c_uint8)),
        ("n_rms", c_uint64), ("n_rms_window", c_uint64), ("n_cells", c_uint64), ("fft_nlogn", c_double),
    ]


def _load() -> ctypes.CDLL:
    if not LIB_PATH.is_file() and (HERE / "visqol_oracle.cpp").is_file():
        build()
    lib = ctypes.CDLL(str(LIB_PATH))
    D, I64, SZ = POINTER(c_double), POINTER(c_int64), POINTER(c_size_t)
    sig = {
        "vqo_options_default": (None, [POINTER(Options)]),
        "vqo_measure": (c_int, [POINTER(Options), D, c_size_t, D, c_size_t, c_uint32,
                                POINTER(POINTER(Result)), POINTER(POINTER(Trace))]),
        "vqo_result_free": (None, [POINTER(Result)]),
        "vqo_trace_free": (None, [POINTER(Trace)]),
        "vqo_measure_batch": (c_int, [POINTER(Options), c_size_t, POINTER(D), SZ, POINTER(D), SZ, c_uint32,
                                      c_uint32, POINTER(POINTER(Result)), POINTER(c_int32)]),
        "vqo_last_error": (c_char_p, []),
        "vqo_uniform_center_freqs": (None, [c_size_t, c_double, c_double, D]),
        "vqo_filters": (None, [c_size_t, c_uint32, c_double, c_double, D, D]),
        "vqo_hann": (None, [c_size_t, D]),
        "vqo_filter_band": (None, [D, D, c_size_t, D]),
        "vqo_filter_band_rms_fresh": (c_double, [D, D, c_size_t]),
        "vqo_spectrogram": (c_size_t, [c_size_t, D, D, c_size_t, c_size_t, D, c_size_t, D]),
        "vqo_upper_envelope": (None, [D, c_size_t, D]),
        "vqo_fft_size_for": (c_size_t, [c_size_t]),
        "vqo_fft_dif": (None, [D, c_size_t]),
        "vqo_fft_dit": (None, [D, c_size_t]),
        "vqo_fft_twiddles": (None, [c_size_t, D]),
        "vqo_best_lag": (c_int64, [D, c_size_t, D, c_size_t]),
        "vqo_envelope_lag": (c_int64, [D, c_size_t, D, c_size_t]),
        "vqo_convert_to_db": (None, [D, c_size_t, c_double]),
        "vqo_raise_floor_per_frame": (None, [D, D, c_size_t, c_size_t, c_size_t, c_double]),
        "vqo_subtract_joint_minimum": (None, [D, c_size_t, D, c_size_t]),
        "vqo_prepare_for_comparison": (None, [D, D, c_size_t, c_size_t, c_size_t]),
        "vqo_conv2d3x3": (None, [D, D, c_size_t, c_size_t]),
        "vqo_patch_similarity": (c_double, [D, D, c_size_t, c_size_t, D, D, D]),
        "vqo_similarity_scalar": (c_double, [D, D, c_size_t, c_size_t]),
        "vqo_nsim_table": (None, [D, c_size_t, D, c_size_t, c_size_t, c_size_t, c_size_t, I64, I64, I64, D]),
        "vqo_dp_backtrack": (c_size_t, [D, c_size_t, c_size_t, I64, I64, I64, POINTER(c_uint8)]),
        "vqo_ref_patch_indices": (c_int, [c_size_t, c_size_t, I64, SZ]),
        "vqo_vad_patch_indices": (c_int, [D, c_size_t, c_size_t, c_size_t, c_size_t, c_double, I64, SZ]),
        "vqo_calc_max_num_patches": (c_size_t, [I64, c_size_t, c_size_t, c_size_t]),
        "vqo_slice_layout": (None, [c_size_t, c_uint32, c_double, c_double, I64, I64, I64]),
        "vqo_trim_geometry": (None, [c_size_t, c_size_t, c_int64, c_uint32, I64, I64, I64, D]),
        "vqo_truncate_aligned": (c_size_t, [D, c_size_t, D, c_size_t, c_int64, c_uint32, D, D]),
        "vqo_spl": (c_double, [D, c_size_t]),
        "vqo_pow": (c_double, [c_double, c_double]),
        "vqo_svr_predict": (c_int, [c_char_p, D, c_size_t, D]),
        "vqo_svr_predict_text": (c_int, [c_char_p, c_size_t, D, c_size_t, D]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def _d(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_double))


def _i64(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_int64))


def f64(x) -> np.ndarray:
    return np.ascontiguousarray(x, dtype=np.float64)


def options(mode: int = 0, radius: int = 60, lattice: bool = False, unscaled: bool = False,
            disable_global_alignment: bool = False, disable_realignment: bool = False,
            model_path: str | None = None) -> Options:
    o = Options()
    lib.vqo_options_default(ctypes.byref(o))
    o.mode, o.search_window_radius = mode, radius
    o.use_lattice_model, o.use_unscaled_speech_mos_mapping = int(lattice), int(unscaled)
    o.disable_global_alignment, o.disable_realignment = int(disable_global_alignment), int(disable_realignment)
    o.model_path = os.fsencode(model_path) if model_path else None
    return o


def _vec(ptr, n):
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0)


def result_dict(r: Result) -> dict:
    nb, npch = r.num_bands, r.num_patches
    patches = []
    for i in range(npch):
        p = r.patch_sims[i]
        patches.append({
            "similarity": p.similarity, "ref_patch_start_time": p.ref_patch_start_time,
            "ref_patch_end_time": p.ref_patch_end_time, "deg_patch_start_time": p.deg_patch_start_time,
            "deg_patch_end_time": p.deg_patch_end_time, "freq_band_means": _vec(p.freq_band_means, nb),
            "freq_band_stddevs": _vec(p.freq_band_stddevs, nb), "freq_band_deg_energy": _vec(p.freq_band_deg_energy, nb),
        })
    return {
        "moslqo": r.moslqo, "vnsim": r.vnsim, "alignment_lag_s": r.alignment_lag_s, "num_bands": nb,
        "fvnsim": _vec(r.fvnsim, nb), "fvnsim10": _vec(r.fvnsim10, nb), "fstdnsim": _vec(r.fstdnsim, nb),
        "fvdegenergy": _vec(r.fvdegenergy, nb), "center_freq_bands": _vec(r.center_freq_bands, nb),
        "patch_sims": patches,
    }


def trace_dict(t: Trace) -> dict:
    n = t.num_patches
    return {
        "global_lag": t.global_lag, "spl_factor": t.spl_factor, "deg_len": t.deg_len,
        "nf_ref": t.nf_ref, "nf_deg": t.nf_deg, "num_patches": n,
        "ref_index": _vec(t.ref_index, n).astype(np.int64) if n else np.zeros(0, np.int64),
        "deg_offset": np.ctypeslib.as_array(t.deg_offset, shape=(n,)).copy() if n else np.zeros(0, np.int64),
        "valid": np.ctypeslib.as_array(t.valid, shape=(n,)).copy() if n else np.zeros(0, np.uint8),
        "realign_lag": np.ctypeslib.as_array(t.realign_lag, shape=(n,)).copy() if n else np.zeros(0, np.int64),
        "realign_frames": np.ctypeslib.as_array(t.realign_frames, shape=(n,)).copy() if n else np.zeros(0, np.int64),
        "realign_reused": np.ctypeslib.as_array(t.realign_reused, shape=(n,)).copy() if n else np.zeros(0, np.uint8),
        "realign_accepted": np.ctypeslib.as_array(t.realign_accepted, shape=(n,)).copy() if n else np.zeros(0, np.uint8),
        "n_rms": t.n_rms, "n_rms_window": t.n_rms_window, "n_cells": t.n_cells, "fft_nlogn": t.fft_nlogn,
    }


class OracleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (code {code})")
        self.code = code


def measure(ref, deg, sample_rate: int, opts: Options | None = None, trace: bool = True):
    """One pair through the oracle: (result dict, trace dict or None)."""
    ref, deg = f64(ref), f64(deg)
    o = opts or options()
    out = POINTER(Result)()
    tr = POINTER(Trace)()
    rc = lib.vqo_measure(ctypes.byref(o), _d(ref), ref.size, _d(deg), deg.size, sample_rate,
                         ctypes.byref(out), ctypes.byref(tr) if trace else None)
    if rc != 0:
        raise OracleError(rc, lib.vqo_last_error().decode())
    try:
        res = result_dict(out.contents)
        t = trace_dict(tr.contents) if trace else None
    finally:
        lib.vqo_result_free(out)
        if trace:
            lib.vqo_trace_free(tr)
    return res, t


def measure_batch(refs, degs, sample_rate: int, opts: Options | None = None, threads: int = 0):
    """Pair-parallel batch on `threads` host threads: list of (code, result dict or None)."""
    n = len(refs)
    refs = [f64(r) for r in refs]
    degs = [f64(d) for d in degs]
    o = opts or options()
    rp = (POINTER(c_double) * n)(*[_d(a) for a in refs])
    dp = (POINTER(c_double) * n)(*[_d(a) for a in degs])
    rl = (c_size_t * n)(*[a.size for a in refs])
    dl = (c_size_t * n)(*[a.size for a in degs])
    outs = (POINTER(Result) * n)()
    st = (c_int32 * n)()
    lib.vqo_measure_batch(ctypes.byref(o), n, rp, rl, dp, dl, sample_rate, threads, outs, st)
    res = []
    for i in range(n):
        if st[i] == 0:
            res.append((0, result_dict(outs[i].contents)))
            lib.vqo_result_free(outs[i])
        else:
            res.append((st[i], None))
    return res


# ---- stage helpers ---------------------------------------------------

def filters(nb: int, sample_rate: int, low: float = 50.0, high: float | None = None):
    coeffs = np.zeros(nb * 8)
    cf = np.zeros(nb)
    lib.vqo_filters(nb, sample_rate, low, high if high is not None else sample_rate / 2.0, _d(coeffs), _d(cf))
    return coeffs.reshape(nb, 8), cf


def hann(size: int) -> np.ndarray:
    out = np.zeros(size)
    lib.vqo_hann(size, _d(out))
    return out


def window_hop(sample_rate: int) -> tuple[int, int]:
    """ensureCache's window and hop (src/visqol.zig:350-352)."""
    import math
    w = int(math.floor(sample_rate * 0.08 + 0.5))
    h = max(1, int(w * 0.25))
    return w, h


def spectrogram(x, coeffs: np.ndarray, window: int, hop: int) -> np.ndarray:
    x = f64(x)
    nb = coeffs.shape[0]
    nf = 0 if x.size < window else 1 + (x.size - window) // hop
    out = np.zeros(nb * max(nf, 1))
    c = f64(coeffs.reshape(-1))
    h = hann(window)
    lib.vqo_spectrogram(nb, _d(c), _d(h), window, hop, _d(x), x.size, _d(out))
    return out[: nb * nf].reshape(nb, nf)


def upper_envelope(x) -> np.ndarray:
    x = f64(x)
    out = np.zeros(x.size)
    lib.vqo_upper_envelope(_d(x), x.size, _d(out))
    return out


def best_lag(a, b) -> int:
    a, b = f64(a), f64(b)
    return int(lib.vqo_best_lag(_d(a), a.size, _d(b), b.size))


def envelope_lag(a, b) -> int:
    a, b = f64(a), f64(b)
    return int(lib.vqo_envelope_lag(_d(a), a.size, _d(b), b.size))


def fft_dif(z: np.ndarray) -> np.ndarray:
    buf = np.ascontiguousarray(z, dtype=np.complex128).copy()
    lib.vqo_fft_dif(buf.ctypes.data_as(POINTER(c_double)), buf.size)
    return buf


def fft_dit(z: np.ndarray) -> np.ndarray:
    buf = np.ascontiguousarray(z, dtype=np.complex128).copy()
    lib.vqo_fft_dit(buf.ctypes.data_as(POINTER(c_double)), buf.size)
    return buf


def convert_to_db(x, floor_db: float) -> np.ndarray:
    x = f64(x).copy()
    lib.vqo_convert_to_db(_d(x), x.size, floor_db)
    return x


def prepare_for_comparison(ref: np.ndarray, deg: np.ndarray):
    r = f64(ref).copy()
    d = f64(deg).copy()
    nb = r.shape[0]
    lib.vqo_prepare_for_comparison(_d(r), _d(d), nb, r.shape[1], d.shape[1])
    return r, d


def conv2d3x3(x: np.ndarray) -> np.ndarray:
    x = f64(x)
    out = np.zeros_like(x)
    lib.vqo_conv2d3x3(_d(x), _d(out), x.shape[0], x.shape[1])
    return out


def patch_similarity(ref: np.ndarray, deg: np.ndarray):
    ref, deg = f64(ref), f64(deg)
    nr, nc = ref.shape
    means, sd, en = np.zeros(nr), np.zeros(nr), np.zeros(nr)
    mean = lib.vqo_patch_similarity(_d(ref), _d(deg), nr, nc, _d(means), _d(sd), _d(en))
    return mean, means, sd, en


def similarity_scalar(ref: np.ndarray, deg: np.ndarray) -> float:
    ref, deg = f64(ref), f64(deg)
    return lib.vqo_similarity_scalar(_d(ref), _d(deg), ref.shape[0], ref.shape[1])


def nsim_table(ref_spec: np.ndarray, deg_spec: np.ndarray, patch: int, ref_idx, lo, hi) -> np.ndarray:
    ref_spec, deg_spec = f64(ref_spec), f64(deg_spec)
    nb, nfr = ref_spec.shape
    nfd = deg_spec.shape[1]
    ri = np.ascontiguousarray(ref_idx, dtype=np.int64)
    lo = np.ascontiguousarray(lo, dtype=np.int64)
    hi = np.ascontiguousarray(hi, dtype=np.int64)
    out = np.zeros(ri.size * nfd)
    lib.vqo_nsim_table(_d(ref_spec), nfr, _d(deg_spec), nfd, nb, patch, ri.size, _i64(ri), _i64(lo), _i64(hi), _d(out))
    return out.reshape(ri.size, nfd)


def dp_backtrack(sims: np.ndarray, lo, hi):
    sims = f64(sims)
    np_, nfd = sims.shape
    lo = np.ascontiguousarray(lo, dtype=np.int64)
    hi = np.ascontiguousarray(hi, dtype=np.int64)
    off = np.zeros(np_, np.int64)
    valid = np.zeros(np_, np.uint8)
    reached = lib.vqo_dp_backtrack(_d(sims), np_, nfd, _i64(lo), _i64(hi), _i64(off),
                                   valid.ctypes.data_as(POINTER(c_uint8)))
    return off, valid, reached


def ref_patch_indices(nf: int, patch: int):
    out = np.zeros(max(nf, 1), np.int64)
    n = c_size_t()
    rc = lib.vqo_ref_patch_indices(nf, patch, _i64(out), ctypes.byref(n))
    if rc != 0:
        raise OracleError(rc, "ReferenceSpectrogramTooSmall")
    return out[: n.value]


def vad_patch_indices(ref, nf: int, patch: int, window: int, overlap: float = 0.25):
    ref = f64(ref)
    out = np.zeros(max(nf, 1), np.int64)
    n = c_size_t()
    lib.vqo_vad_patch_indices(_d(ref), ref.size, nf, patch, window, overlap, _i64(out), ctypes.byref(n))
    return out[: n.value]


def calc_max_num_patches(idx, nf_deg: int, patch: int) -> int:
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    return int(lib.vqo_calc_max_num_patches(_i64(idx), idx.size, nf_deg, patch))


def slice_layout(length: int, sr: int, t0: float, t1: float):
    pad, base, n = c_int64(), c_int64(), c_int64()
    lib.vqo_slice_layout(length, sr, t0, t1, ctypes.byref(pad), ctypes.byref(base), ctypes.byref(n))
    return pad.value, base.value, n.value


def trim_geometry(ref_len: int, deg_len: int, lag: int, sr: int):
    ln, ro, do, ls = c_int64(), c_int64(), c_int64(), c_double()
    lib.vqo_trim_geometry(ref_len, deg_len, lag, sr, ctypes.byref(ln), ctypes.byref(ro), ctypes.byref(do), ctypes.byref(ls))
    return ln.value, ro.value, do.value, ls.value


def truncate_aligned(ref, deg, lag: int, sr: int):
    ref, deg = f64(ref), f64(deg)
    ro = np.zeros(max(ref.size, 1))
    do = np.zeros(max(ref.size, 1))
    n = lib.vqo_truncate_aligned(_d(ref), ref.size, _d(deg), deg.size, lag, sr, _d(ro), _d(do))
    return ro[:n], do[:n]


def spl(x) -> float:
    x = f64(x)
    return lib.vqo_spl(_d(x), x.size)


def zig_pow(x: float, y: float) -> float:
    return lib.vqo_pow(x, y)


def svr_predict(x, model_text: str | None = None) -> float:
    x = f64(x)
    y = c_double()
    if model_text is None:
        rc = lib.vqo_svr_predict(None, _d(x), x.size, ctypes.byref(y))
    else:
        t = model_text.encode()
        rc = lib.vqo_svr_predict_text(t, len(t), _d(x), x.size, ctypes.byref(y))
    if rc != 0:
        raise OracleError(rc, lib.vqo_last_error().decode())
    return y.value
