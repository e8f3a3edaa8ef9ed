"""ctypes binding of libvisqol (include/visqol.h + include/visqol_b200.h).

The ABI's structures (``Options``, ``Patch``, ``Result``; their layouts are
fixed by include/visqol.h, as in the reference's src/include/visqol.h) and a
``Context`` over one ``visqol_ctx`` with scoring of pairs, batches and WAV
files, plus this library's extensions: traced batches (per-pair lags and
matches), device-resident inputs, prepared references, the request server,
per-stage timing, and single-stage calls. The reference's own Python
package binds the same ABI with its own module and loads this library
unchanged.

There is no fallback: if ``libvisqol.so`` is missing, importing this module
raises ImportError.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import (POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_size_t, c_uint8, c_uint32,
                    c_uint64, c_void_p)
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libvisqol.so"

MODE_AUDIO = 0
MODE_SPEECH = 1
BACKENDS = {"cpu": 0, "metal": 1, "cuda": 2, "vulkan": 3}
PRECISIONS = {"exact": 0, "fast": 1, "balanced": 2, "auto": 3}

OK = 0
E_INVALID_ARGUMENT = -1
E_OUT_OF_MEMORY = -2
E_IO = -3
E_MODEL = -4
E_SIGNAL = -5
E_BACKEND = -6
E_INTERNAL = -7

DEVICE_INPUTS = 1


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


class Timing(ctypes.Structure):
    _fields_ = [
        ("total_ms", c_double), ("lag_ms", c_double), ("spectrogram_ms", c_double), ("prep_ms", c_double),
        ("nsim_ms", c_double), ("realign_ms", c_double), ("gammatone_kernel_ms", c_double),
        ("gammatone_launches", c_uint64), ("gammatone_rms", c_uint64), ("gammatone_window", c_uint64),
        ("kernel_launches", c_uint64), ("h2d_bytes", c_uint64), ("d2h_bytes", c_uint64), ("host_syncs", c_uint64),
        ("lag_kernel_ms", c_double), ("lag_bytes", c_uint64), ("lag_reruns", c_uint64),
    ]


class ServeConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", c_uint64), ("lanes", c_uint32), ("max_batch", c_uint32)]


class ServeStats(ctypes.Structure):
    _fields_ = [
        ("submitted", c_uint64), ("completed", c_uint64), ("failed", c_uint64), ("queued", c_uint64),
        ("in_flight", c_uint64), ("batches", c_uint64), ("hbm_budget_bytes", c_uint64),
        ("hbm_in_flight_bytes", c_uint64), ("hbm_reserved_bytes", c_uint64),
        ("latency_p50_ms", c_double), ("latency_p99_ms", c_double), ("latency_mean_ms", c_double),
        ("queue_p50_ms", c_double), ("queue_p99_ms", c_double), ("mean_batch", c_double),
    ]


def build() -> Path:
    """Compile libvisqol.so with the package Makefile (no-op when current)."""
    subprocess.run(["make", "-s", "-j8", "-C", str(HERE)], check=True)
    return LIB_PATH


def _load() -> ctypes.CDLL:
    override = os.environ.get("VISQOL_B200_LIBRARY")
    path = Path(override) if override else LIB_PATH
    if not path.is_file():
        raise ImportError(f"libvisqol not found at {path}; build it with `make -C {HERE}`")
    lib = ctypes.CDLL(str(path))
    D, I64, SZ, U8 = POINTER(c_double), POINTER(c_int64), POINTER(c_size_t), POINTER(c_uint8)
    sig = {
        "visqol_abi_version": (c_uint32, []),
        "visqol_version": (c_char_p, []),
        "visqol_last_error": (c_char_p, []),
        "visqol_available_backends": (c_uint32, []),
        "visqol_options_default": (None, [POINTER(Options)]),
        "visqol_create": (c_int, [POINTER(Options), POINTER(c_void_p)]),
        "visqol_destroy": (None, [c_void_p]),
        "visqol_measure": (c_int, [c_void_p, D, c_size_t, D, c_size_t, c_uint32, POINTER(POINTER(Result))]),
        "visqol_measure_files": (c_int, [c_void_p, c_char_p, c_char_p, POINTER(POINTER(Result))]),
        "visqol_measure_batch": (c_int, [c_void_p, c_size_t, POINTER(c_void_p), SZ, POINTER(c_void_p), SZ, c_uint32,
                                         c_uint32, POINTER(POINTER(Result)), POINTER(c_int32)]),
        "visqol_measure_files_batch": (c_int, [c_void_p, c_size_t, POINTER(c_char_p), POINTER(c_char_p), c_uint32,
                                               POINTER(POINTER(Result)), POINTER(c_int32)]),
        "visqol_result_free": (None, [POINTER(Result)]),
        "visqol_b200_measure_batch": (c_int, [c_void_p, c_size_t, POINTER(c_void_p), SZ, POINTER(c_void_p), SZ,
                                              c_uint32, c_uint32, POINTER(POINTER(Result)), POINTER(c_int32),
                                              POINTER(POINTER(Trace))]),
        "visqol_b200_measure_batch_grad": (c_int, [c_void_p, c_size_t, POINTER(c_void_p), SZ, POINTER(c_void_p), SZ,
                                                   c_uint32, c_uint32, POINTER(POINTER(Result)), POINTER(c_int32),
                                                   POINTER(c_void_p)]),
        "visqol_b200_trace_free": (None, [POINTER(Trace)]),
        "visqol_b200_last_timing": (c_int, [c_void_p, POINTER(Timing)]),
        "visqol_b200_device_info": (c_int, [c_int, c_char_p, c_size_t, POINTER(c_int), POINTER(c_int),
                                            POINTER(c_int)]),
        "visqol_b200_spectrogram": (c_int, [c_size_t, D, D, c_size_t, c_size_t, D, c_size_t, D, SZ]),
        "visqol_b200_envelope_lag": (c_int, [D, c_size_t, D, c_size_t, I64]),
        "visqol_b200_best_lag": (c_int, [D, c_size_t, D, c_size_t, I64]),
        "visqol_b200_signal_sums": (c_int, [D, c_size_t, c_size_t, D]),
        "visqol_b200_lag_search": (c_int, [D, c_size_t, D, c_size_t, c_int, c_int, I64, POINTER(c_int32),
                                           POINTER(c_float), c_size_t]),
        "visqol_b200_refine_lag": (c_int, [D, c_size_t, D, c_size_t, POINTER(c_float), c_size_t, c_double, c_double,
                                           I64, POINTER(c_int32)]),
        "visqol_b200_fft": (c_int, [D, c_size_t, c_int]),
        "visqol_b200_nsim_quotient": (c_int, [D, D, c_size_t, D]),
        "visqol_b200_patch_similarity_grad": (c_int, [D, D, c_size_t, c_size_t, D, D, D, D, D]),
        "visqol_b200_prepare_grad": (c_int, [D, D, c_size_t, c_size_t, c_size_t, D, D, D]),
        "visqol_b200_prepare_for_comparison": (c_int, [D, D, c_size_t, c_size_t, c_size_t]),
        "visqol_b200_log10": (c_int, [D, c_size_t, D]),
        "visqol_b200_nsim_table": (c_int, [D, c_size_t, D, c_size_t, c_size_t, c_size_t, c_size_t, I64, I64, I64, D]),
        "visqol_b200_dp": (c_int, [D, c_size_t, c_size_t, I64, I64, I64, U8, SZ]),
        "visqol_b200_dp_static": (c_int, [D, c_size_t, c_size_t, I64, I64, I64, U8, SZ]),
        "visqol_b200_patch_similarity": (c_int, [D, D, c_size_t, c_size_t, D, D, D, D]),
        "visqol_b200_peak": (c_int, [c_int, D]),
        "visqol_b200_autotune_choices": (c_int, [POINTER(c_int32), c_size_t, SZ]),
        "visqol_b200_lattice_predict": (c_int, [c_char_p, c_size_t, D, D, D, D, D]),
        "visqol_b200_prepare": (c_int, [c_void_p, c_size_t, POINTER(c_void_p), SZ, c_uint32, c_uint32,
                                        POINTER(c_void_p)]),
        "visqol_b200_measure_prepared": (c_int, [c_void_p, c_void_p, c_size_t, SZ, POINTER(c_void_p), SZ, c_uint32,
                                                 POINTER(POINTER(Result)), POINTER(c_int32)]),
        "visqol_b200_prepared_free": (None, [c_void_p]),
        "visqol_b200_server_create": (c_int, [POINTER(Options), POINTER(ServeConfig), POINTER(c_void_p)]),
        "visqol_b200_server_destroy": (None, [c_void_p]),
        "visqol_b200_server_submit": (c_int, [c_void_p, c_uint32, c_void_p, c_size_t, c_void_p, c_size_t, c_uint32,
                                              c_uint32, POINTER(c_uint64)]),
        "visqol_b200_server_next": (c_int, [c_void_p, c_int32, POINTER(c_uint64), POINTER(c_int32),
                                            POINTER(POINTER(Result))]),
        "visqol_b200_server_stats": (c_int, [c_void_p, POINTER(ServeStats), c_int]),
        "visqol_b200_pair_footprint": (c_int, [c_size_t, c_size_t, c_uint32, c_uint32, POINTER(c_uint64)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()

ABI_VERSION = 1
if lib.visqol_abi_version() != ABI_VERSION:
    raise ImportError(f"libvisqol ABI {lib.visqol_abi_version()} does not match the bindings ({ABI_VERSION})")

__version__ = lib.visqol_version().decode()

# Every symbol include/visqol.h and include/visqol_b200.h declare.
EXPORTS = [
    "visqol_abi_version", "visqol_version", "visqol_last_error", "visqol_available_backends",
    "visqol_options_default", "visqol_create", "visqol_destroy", "visqol_measure", "visqol_measure_files",
    "visqol_measure_batch", "visqol_measure_files_batch", "visqol_result_free",
    "visqol_b200_measure_batch", "visqol_b200_measure_batch_grad", "visqol_b200_trace_free", "visqol_b200_last_timing", "visqol_b200_device_info",
    "visqol_b200_spectrogram", "visqol_b200_envelope_lag", "visqol_b200_best_lag", "visqol_b200_fft",
    "visqol_b200_signal_sums",
    "visqol_b200_lag_search", "visqol_b200_refine_lag", "visqol_b200_nsim_quotient",
    "visqol_b200_patch_similarity_grad", "visqol_b200_prepare_grad",
    "visqol_b200_prepare_for_comparison", "visqol_b200_log10", "visqol_b200_nsim_table", "visqol_b200_dp",
    "visqol_b200_dp_static",
    "visqol_b200_patch_similarity", "visqol_b200_peak",
    "visqol_b200_lattice_predict", "visqol_b200_autotune_choices",
    "visqol_b200_prepare", "visqol_b200_measure_prepared", "visqol_b200_prepared_free",
    "visqol_b200_server_create", "visqol_b200_server_destroy", "visqol_b200_server_submit",
    "visqol_b200_server_next", "visqol_b200_server_stats", "visqol_b200_pair_footprint",
]


# Status names of include/visqol.h, for messages.
_STATUS = {OK: "OK", E_INVALID_ARGUMENT: "INVALID_ARGUMENT", E_OUT_OF_MEMORY: "OUT_OF_MEMORY", E_IO: "IO",
           E_MODEL: "MODEL", E_SIGNAL: "SIGNAL", E_BACKEND: "BACKEND", E_INTERNAL: "INTERNAL"}


class NativeError(RuntimeError):
    """A non-zero status from libvisqol: ``code`` is the negative status of
    include/visqol.h; the message is the library's text for the failure."""

    def __init__(self, code: int, message: str):
        self.code = int(code)
        super().__init__(f"{_STATUS.get(self.code, self.code)}: {message}")


def error_for(code: int) -> NativeError:
    """`code` with the calling thread's last library message."""
    text = lib.visqol_last_error()
    return NativeError(code, text.decode("utf-8", "replace") if text else "")


def _check(rc: int) -> None:
    if rc:
        raise error_for(rc)


def available_backends() -> list[str]:
    """Backends this library runs, by name (its bit mask)."""
    mask = int(lib.visqol_available_backends())
    return [b for b, bit in sorted(BACKENDS.items(), key=lambda kv: kv[1]) if mask >> bit & 1]


def mono(x, what: str = "signal") -> np.ndarray:
    """x as contiguous float64 samples; copies only when it must."""
    arr = np.ascontiguousarray(x, dtype=np.float64)
    if arr.ndim != 1:
        raise ValueError(f"{what}: mono samples expected (a 1-D array), not shape {arr.shape}")
    return arr


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_double))


def _i64(a: np.ndarray):
    return a.ctypes.data_as(POINTER(c_int64))


class _Signals:
    """A batch's signal table as the C calls take it: an array of sample
    pointers and one of lengths. Host signals are converted to float64 and
    held here for the call's lifetime; device signals are addresses (ints)
    with their lengths."""

    def __init__(self, signals, lengths=None, device: bool = False):
        n = len(signals)
        if device:
            if lengths is None or len(lengths) != n:
                raise ValueError("device signals need one length each")
            self.hold = ()
            addrs, counts = [int(p) for p in signals], [int(c) for c in lengths]
        else:
            self.hold = [mono(x) for x in signals]
            addrs, counts = [a.ctypes.data for a in self.hold], [a.size for a in self.hold]
        self.ptrs = (c_void_p * n)(*addrs)
        self.lens = (c_size_t * n)(*counts)


def _outcomes(outs, status, n: int) -> list:
    """Per pair: its Result pointer, or a NativeError with its status."""
    got = []
    for i in range(n):
        code = int(status[i])
        got.append(outs[i] if code == OK else NativeError(code, f"pair {i} failed"))
    return got


# Context keyword -> (Options field, conversion)
_OPTION_FIELDS = {
    "mode": ("mode", int),
    "search_window_radius": ("search_window_radius", int),
    "use_unscaled_speech_mos_mapping": ("use_unscaled_speech_mos_mapping", lambda v: int(bool(v))),
    "disable_global_alignment": ("disable_global_alignment", lambda v: int(bool(v))),
    "disable_realignment": ("disable_realignment", lambda v: int(bool(v))),
    "use_lattice_model": ("use_lattice_model", lambda v: int(bool(v))),
}


def make_options(backend: str = "cuda", precision: str | None = None, model_path: str | None = None,
                 **settings) -> Options:
    """visqol_options from the library defaults, overridden by keyword."""
    if backend not in BACKENDS:
        raise ValueError(f"backend {backend!r} is none of {', '.join(sorted(BACKENDS))}")
    if precision is not None and precision not in PRECISIONS:
        raise ValueError(f"precision {precision!r} is none of {', '.join(sorted(PRECISIONS))}")
    opts = Options()
    lib.visqol_options_default(ctypes.byref(opts))
    for key, value in settings.items():
        if key not in _OPTION_FIELDS:
            raise TypeError(f"unknown option {key!r}")
        field, conv = _OPTION_FIELDS[key]
        setattr(opts, field, conv(value))
    opts.model_path = os.fsencode(model_path) if model_path else None
    opts.backend = BACKENDS[backend]
    if precision is not None:
        opts.precision = PRECISIONS[precision]
    return opts


class Context:
    """A ``visqol_ctx``: options fixed at creation, one thread at a time.

    Scoring calls return ``Result`` pointers (free them with ``free``), and
    batch calls a list with a ``NativeError`` in place of each failed pair.
    """

    def __init__(self, *, mode: int = MODE_AUDIO, search_window_radius: int = 60,
                 use_unscaled_speech_mos_mapping: bool = False, disable_global_alignment: bool = False,
                 disable_realignment: bool = False, use_lattice_model: bool = False, model_path: str | None = None,
                 backend: str = "cuda", precision: str | None = None):
        opts = make_options(backend, precision, model_path, mode=mode, search_window_radius=search_window_radius,
                            use_unscaled_speech_mos_mapping=use_unscaled_speech_mos_mapping,
                            disable_global_alignment=disable_global_alignment,
                            disable_realignment=disable_realignment, use_lattice_model=use_lattice_model)
        handle = c_void_p()
        _check(lib.visqol_create(ctypes.byref(opts), ctypes.byref(handle)))
        self._handle = handle

    def close(self) -> None:
        handle, self._handle = getattr(self, "_handle", None), None
        if handle:
            lib.visqol_destroy(handle)

    def __del__(self):
        self.close()

    def measure(self, ref, deg, sample_rate: int):
        ref, deg = mono(ref, "ref"), mono(deg, "deg")
        out = POINTER(Result)()
        _check(lib.visqol_measure(self._handle, _dptr(ref), ref.size, _dptr(deg), deg.size, sample_rate,
                                  ctypes.byref(out)))
        return out

    def measure_files(self, ref_path: str, deg_path: str):
        out = POINTER(Result)()
        _check(lib.visqol_measure_files(self._handle, os.fsencode(ref_path), os.fsencode(deg_path),
                                        ctypes.byref(out)))
        return out

    def _pairs_call(self, fn, n: int, *args):
        outs, status = (POINTER(Result) * n)(), (c_int32 * n)()
        rc = fn(self._handle, n, *args, outs, status)
        if rc and all(int(status[i]) == OK for i in range(n)):
            raise error_for(rc)  # the call itself was refused
        return _outcomes(outs, status, n)

    def measure_batch(self, refs, degs, sample_rate: int, num_threads: int = 0):
        r, d = _Signals(refs), _Signals(degs)
        return self._pairs_call(lib.visqol_measure_batch, len(refs), r.ptrs, r.lens, d.ptrs, d.lens, sample_rate,
                                num_threads)

    def measure_files_batch(self, ref_paths, deg_paths, num_threads: int = 0):
        n = len(ref_paths)
        enc = lambda paths: (c_char_p * n)(*map(os.fsencode, paths))  # noqa: E731
        return self._pairs_call(lib.visqol_measure_files_batch, n, enc(ref_paths), enc(deg_paths), num_threads)

    def prepare(self, refs, sample_rate: int, device_inputs: bool = False, ref_lens=None) -> "Prepared":
        """Reference-side work for scoring many degraded signals against
        these references (visqol_b200_prepare)."""
        return Prepared(self, refs, sample_rate, device_inputs, ref_lens)

    def measure_prepared(self, prepared: "Prepared", degs, ref_index=None, device_inputs: bool = False,
                         deg_lens=None):
        """degs[i] against prepared reference ref_index[i] (default i), as
        measure_batch."""
        n = len(degs)
        d = _Signals(degs, deg_lens, device_inputs)
        ix = (c_size_t * n)(*ref_index) if ref_index is not None else None
        flags = DEVICE_INPUTS if device_inputs else 0
        outs, status = (POINTER(Result) * n)(), (c_int32 * n)()
        rc = lib.visqol_b200_measure_prepared(self._handle, prepared._handle, n, ix, d.ptrs, d.lens, flags, outs,
                                              status)
        if rc and all(int(status[i]) == OK for i in range(n)):
            raise error_for(rc)
        return _outcomes(outs, status, n)

    def _b200_batch(self, refs, degs, sample_rate, device_inputs, ref_lens, deg_lens, traces):
        n = len(refs)
        r = _Signals(refs, ref_lens, device_inputs)
        d = _Signals(degs, deg_lens, device_inputs)
        outs, status = (POINTER(Result) * n)(), (c_int32 * n)()
        lib.visqol_b200_measure_batch(self._handle, n, r.ptrs, r.lens, d.ptrs, d.lens, sample_rate,
                                      DEVICE_INPUTS if device_inputs else 0, outs, status, traces)
        return outs, status

    def measure_batch_scores(self, refs, degs, sample_rate: int, device_inputs: bool = False,
                             ref_lens=None, deg_lens=None):
        """Batch without traces: ``(code, MOS or None)`` per pair (the
        results are freed here)."""
        outs, status = self._b200_batch(refs, degs, sample_rate, device_inputs, ref_lens, deg_lens, None)
        scores = []
        for i in range(len(refs)):
            if int(status[i]) == OK:
                scores.append((OK, outs[i].contents.moslqo))
                free(outs[i])
            else:
                scores.append((int(status[i]), None))
        return scores

    def measure_batch_traced(self, refs, degs, sample_rate: int, device_inputs: bool = False,
                             ref_lens=None, deg_lens=None):
        """Batch with per-pair traces. Host arrays, or device addresses (ints)
        with their lengths when ``device_inputs``. Returns a list of
        ``(code, result dict or None, trace dict or None)``."""
        traces = (POINTER(Trace) * len(refs))()
        outs, status = self._b200_batch(refs, degs, sample_rate, device_inputs, ref_lens, deg_lens, traces)
        got = []
        for i in range(len(refs)):
            if int(status[i]) == OK:
                got.append((OK, result_dict(outs[i].contents), trace_dict(traces[i].contents)))
                free(outs[i])
                lib.visqol_b200_trace_free(traces[i])
            else:
                got.append((int(status[i]), None, None))
        return got

    def measure_batch_grad(self, refs, degs, sample_rate: int):
        """Scores with d moslqo / d degraded signal: per pair ``(code,
        result dict or None, gradient array or None)``."""
        n = len(refs)
        r, d = _Signals(refs), _Signals(degs)
        grads = [np.zeros(a.size) for a in d.hold]
        gp = (c_void_p * n)(*[g.ctypes.data for g in grads])
        outs, status = (POINTER(Result) * n)(), (c_int32 * n)()
        rc = lib.visqol_b200_measure_batch_grad(self._handle, n, r.ptrs, r.lens, d.ptrs, d.lens, sample_rate, 0, outs,
                                                status, gp)
        if rc and all(int(status[i]) == OK for i in range(n)):
            raise error_for(rc)
        got = []
        for i in range(n):
            if int(status[i]) == OK:
                got.append((OK, result_dict(outs[i].contents), grads[i]))
                free(outs[i])
            else:
                got.append((int(status[i]), None, None))
        return got

    def last_timing(self) -> dict:
        t = Timing()
        _check(lib.visqol_b200_last_timing(self._handle, ctypes.byref(t)))
        return {name: getattr(t, name) for name, _ in Timing._fields_}


def free(result) -> None:
    """Release a Result the library returned."""
    lib.visqol_result_free(result)


def vec(ptr, n: int) -> np.ndarray:
    """n doubles at ptr, copied."""
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0)


def result_dict(r: Result) -> dict:
    nb, npch = r.num_bands, r.num_patches
    patches = []
    for i in range(npch):
        p = r.patch_sims[i]
        patches.append({
            "similarity": p.similarity, "ref_patch_start_time": p.ref_patch_start_time,
            "ref_patch_end_time": p.ref_patch_end_time, "deg_patch_start_time": p.deg_patch_start_time,
            "deg_patch_end_time": p.deg_patch_end_time, "freq_band_means": vec(p.freq_band_means, nb),
            "freq_band_stddevs": vec(p.freq_band_stddevs, nb), "freq_band_deg_energy": vec(p.freq_band_deg_energy, nb),
        })
    return {
        "moslqo": r.moslqo, "vnsim": r.vnsim, "alignment_lag_s": r.alignment_lag_s, "num_bands": nb,
        "fvnsim": vec(r.fvnsim, nb), "fvnsim10": vec(r.fvnsim10, nb), "fstdnsim": vec(r.fstdnsim, nb),
        "fvdegenergy": vec(r.fvdegenergy, nb), "center_freq_bands": vec(r.center_freq_bands, nb),
        "patch_sims": patches,
    }


def _arr(ptr, n, dtype):
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0, dtype)


def trace_dict(t: Trace) -> dict:
    n = t.num_patches
    return {
        "global_lag": t.global_lag, "spl_factor": t.spl_factor, "deg_len": t.deg_len,
        "nf_ref": t.nf_ref, "nf_deg": t.nf_deg, "num_patches": n,
        "ref_index": _arr(t.ref_index, n, np.int64), "deg_offset": _arr(t.deg_offset, n, np.int64),
        "valid": _arr(t.valid, n, np.uint8), "realign_lag": _arr(t.realign_lag, n, np.int64),
        "realign_frames": _arr(t.realign_frames, n, np.int64), "realign_reused": _arr(t.realign_reused, n, np.uint8),
        "realign_accepted": _arr(t.realign_accepted, n, np.uint8),
        "n_rms": t.n_rms, "n_rms_window": t.n_rms_window, "n_cells": t.n_cells, "fft_nlogn": t.fft_nlogn,
    }


def device_info(device: int = 0) -> dict:
    name = ctypes.create_string_buffer(256)
    sm, ma, mi = c_int(), c_int(), c_int()
    _check(lib.visqol_b200_device_info(device, name, 256, ctypes.byref(sm), ctypes.byref(ma), ctypes.byref(mi)))
    return {"name": name.value.decode(), "sm_count": sm.value, "cc": (ma.value, mi.value)}


def peak_tflops(kind: int) -> float:
    """Measured pipe peak: 0 f64 mul/add (no FMA), 1 f64 FMA, 2 f32 FMA."""
    t = c_double()
    _check(lib.visqol_b200_peak(kind, ctypes.byref(t)))
    return t.value


# ---- single-stage calls (exact f64 kernels on host buffers) ----------------

def spectrogram(x, coeffs: np.ndarray, hann: np.ndarray, window: int, hop: int) -> np.ndarray:
    x = mono(x, "x")
    c = np.ascontiguousarray(coeffs, dtype=np.float64).reshape(-1)
    h = np.ascontiguousarray(hann, dtype=np.float64)
    nb = c.size // 8
    nf_max = 0 if x.size < window else 1 + (x.size - window) // hop
    out = np.zeros(max(1, nb * nf_max))
    nf = c_size_t()
    _check(lib.visqol_b200_spectrogram(nb, _dptr(c), _dptr(h), window, hop, _dptr(x), x.size, _dptr(out),
                                       ctypes.byref(nf)))
    return out[: nb * nf.value].reshape(nb, nf.value)


def envelope_lag(a, b) -> int:
    a, b = mono(a, "a"), mono(b, "b")
    lag = c_int64()
    _check(lib.visqol_b200_envelope_lag(_dptr(a), a.size, _dptr(b), b.size, ctypes.byref(lag)))
    return lag.value


def signal_sums(x, skip: int = 0) -> dict:
    """The serial statistics of x as the CPU sums them, bit for bit:
    {"sum", "nyquist", "energy", "first_nonzero", "aligned_energy"} (the
    last over x[skip:]); see visqol_b200_signal_sums."""
    x = mono(x, "x")
    out = np.zeros(5)
    _check(lib.visqol_b200_signal_sums(_dptr(x), x.size, skip, _dptr(out)))
    return {"sum": out[0], "nyquist": out[1], "energy": out[2], "first_nonzero": int(out[3]),
            "aligned_energy": out[4]}


def best_lag(a, b) -> int:
    a, b = mono(a, "a"), mono(b, "b")
    lag = c_int64()
    _check(lib.visqol_b200_best_lag(_dptr(a), a.size, _dptr(b), b.size, ctypes.byref(lag)))
    return lag.value


def lag_search(a, b, raw: bool = False, form: str = "exact", corr: bool = False):
    """One pair's lag by the f64 transform ("exact") or by the f32-nominated
    search the batches run ("fast"):
    (lag, undecided, f32 correlation or None); see visqol_b200_lag_search."""
    a, b = mono(a, "a"), mono(b, "b")
    lag, und = c_int64(), c_int32()
    out, n = None, 0
    if corr:
        n = 1
        while n < 2 * max(a.size, b.size) - 1:
            n <<= 1
        out = np.zeros(n, np.float32)
    code = lib.visqol_b200_lag_search(_dptr(a), a.size, _dptr(b), b.size, int(raw), 1 if form == "fast" else 0,
                                      ctypes.byref(lag), ctypes.byref(und),
                                      out.ctypes.data_as(POINTER(c_float)) if corr else None, n)
    _check(code)
    return lag.value, und.value, out


def refine_lag(s1, s2, approx, scale: float, tol: float):
    """Device refineLag on a caller's approximate correlation: the lag, or
    None where more than 64 lags qualify."""
    s1, s2 = mono(s1, "s1"), mono(s2, "s2")
    approx = np.ascontiguousarray(approx, dtype=np.float32)
    lag, decided = c_int64(), c_int32()
    _check(lib.visqol_b200_refine_lag(_dptr(s1), s1.size, _dptr(s2), s2.size,
                                      approx.ctypes.data_as(POINTER(c_float)), approx.size, scale, tol,
                                      ctypes.byref(lag), ctypes.byref(decided)))
    return lag.value if decided.value else None


def nsim_quotient(num, den) -> np.ndarray:
    """The fast forms' NSIM quotient num / den elementwise on the device."""
    num, den = mono(num, "num"), mono(den, "den")
    if num.size != den.size:
        raise ValueError("num and den differ in length")
    out = np.empty(num.size)
    _check(lib.visqol_b200_nsim_quotient(_dptr(num), _dptr(den), num.size, _dptr(out)))
    return out


def patch_similarity_grad(ref, deg, dmeans=None, dstddevs=None, denergy=None):
    """Host reverse of the patch statistics: (dref, ddeg), each ref.shape."""
    ref = np.ascontiguousarray(ref, dtype=np.float64)
    deg = np.ascontiguousarray(deg, dtype=np.float64)
    nr, nc = ref.shape
    dref, ddeg = np.zeros_like(ref), np.zeros_like(deg)
    opt = [None if v is None else mono(v) for v in (dmeans, dstddevs, denergy)]
    _check(lib.visqol_b200_patch_similarity_grad(_dptr(ref), _dptr(deg), nr, nc,
                                                 *[None if v is None else _dptr(v) for v in opt],
                                                 _dptr(dref), _dptr(ddeg)))
    return dref, ddeg


def prepare_grad(ref_raw, deg_raw, g_ref, g_deg) -> np.ndarray:
    """Host reverse of prepareForComparison: d loss / d raw degraded cells."""
    ref_raw = np.ascontiguousarray(ref_raw, dtype=np.float64)
    deg_raw = np.ascontiguousarray(deg_raw, dtype=np.float64)
    g_ref = np.ascontiguousarray(g_ref, dtype=np.float64)
    g_deg = np.ascontiguousarray(g_deg, dtype=np.float64)
    nb, nfr = ref_raw.shape
    out = np.zeros_like(deg_raw)
    _check(lib.visqol_b200_prepare_grad(_dptr(ref_raw), _dptr(deg_raw), nb, nfr, deg_raw.shape[1], _dptr(g_ref),
                                        _dptr(g_deg), _dptr(out)))
    return out


def fft(z: np.ndarray, inverse: bool = False) -> np.ndarray:
    buf = np.ascontiguousarray(z, dtype=np.complex128).copy()
    _check(lib.visqol_b200_fft(buf.ctypes.data_as(POINTER(c_double)), buf.size, int(inverse)))
    return buf


def prepare_for_comparison(ref: np.ndarray, deg: np.ndarray):
    r = np.ascontiguousarray(ref, dtype=np.float64).copy()
    d = np.ascontiguousarray(deg, dtype=np.float64).copy()
    _check(lib.visqol_b200_prepare_for_comparison(_dptr(r), _dptr(d), r.shape[0], r.shape[1], d.shape[1]))
    return r, d


def log10x10(x) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    _check(lib.visqol_b200_log10(_dptr(x), x.size, _dptr(out)))
    return out


def nsim_table(ref_spec, deg_spec, patch: int, ref_idx, lo, hi) -> np.ndarray:
    rs = np.ascontiguousarray(ref_spec, dtype=np.float64)
    ds = np.ascontiguousarray(deg_spec, dtype=np.float64)
    nb, nfr = rs.shape
    nfd = ds.shape[1]
    ri = np.ascontiguousarray(ref_idx, dtype=np.int64)
    lo = np.ascontiguousarray(lo, dtype=np.int64)
    hi = np.ascontiguousarray(hi, dtype=np.int64)
    out = np.zeros(max(1, ri.size * nfd))
    _check(lib.visqol_b200_nsim_table(_dptr(rs), nfr, _dptr(ds), nfd, nb, patch, ri.size, _i64(ri), _i64(lo),
                                      _i64(hi), _dptr(out)))
    return out[: ri.size * nfd].reshape(ri.size, nfd)


def dp(sims, lo, hi, static_scratch=False):
    """Matched offset, validity and reached count per patch; with
    static_scratch the call goes through visqol_b200_dp_static, which takes
    its device buffers from the library's reserved array."""
    s = np.ascontiguousarray(sims, dtype=np.float64)
    np_, nfd = s.shape
    lo = np.ascontiguousarray(lo, dtype=np.int64)
    hi = np.ascontiguousarray(hi, dtype=np.int64)
    off = np.zeros(np_, np.int64)
    valid = np.zeros(np_, np.uint8)
    reached = c_size_t()
    fn = lib.visqol_b200_dp_static if static_scratch else lib.visqol_b200_dp
    _check(fn(_dptr(s), np_, nfd, _i64(lo), _i64(hi), _i64(off), valid.ctypes.data_as(POINTER(c_uint8)),
              ctypes.byref(reached)))
    return off, valid, reached.value


def patch_similarity(ref, deg):
    r = np.ascontiguousarray(ref, dtype=np.float64)
    d = np.ascontiguousarray(deg, dtype=np.float64)
    nr, nc = r.shape
    means, sd, en, mean = np.zeros(nr), np.zeros(nr), np.zeros(nr), c_double()
    _check(lib.visqol_b200_patch_similarity(_dptr(r), _dptr(d), nr, nc, _dptr(means), _dptr(sd), _dptr(en),
                                            ctypes.byref(mean)))
    return mean.value, means, sd, en


PENDING = 1


def pair_footprint(ref_len: int, deg_len: int, sample_rate: int, mode: int = MODE_AUDIO) -> int:
    """Upper bound of the device memory one pair takes in a batch (bytes)."""
    b = c_uint64()
    _check(lib.visqol_b200_pair_footprint(ref_len, deg_len, sample_rate, mode, ctypes.byref(b)))
    return b.value


class Server:
    """Owns a ``visqol_b200_server``: requests submitted one at a time from
    any thread, scored in continuously refilled batches on the GPU."""

    def __init__(self, *, precision: str = "exact", lanes: int = 0, max_batch: int = 0, hbm_budget_bytes: int = 0,
                 search_window_radius: int = 60, disable_global_alignment: bool = False,
                 disable_realignment: bool = False, use_unscaled_speech_mos_mapping: bool = False):
        opts = Options()
        lib.visqol_options_default(ctypes.byref(opts))
        opts.precision = PRECISIONS[precision]
        opts.search_window_radius = search_window_radius
        opts.disable_global_alignment = int(bool(disable_global_alignment))
        opts.disable_realignment = int(bool(disable_realignment))
        opts.use_unscaled_speech_mos_mapping = int(bool(use_unscaled_speech_mos_mapping))
        opts.use_lattice_model = 0
        cfg = ServeConfig(hbm_budget_bytes, lanes, max_batch)
        handle = c_void_p()
        _check(lib.visqol_b200_server_create(ctypes.byref(opts), ctypes.byref(cfg), ctypes.byref(handle)))
        self._handle = handle

    def close(self) -> None:
        if getattr(self, "_handle", None):
            lib.visqol_b200_server_destroy(self._handle)
            self._handle = None

    def __del__(self):
        self.close()

    def submit(self, mode: int, ref, deg, sample_rate: int, device_inputs: bool = False,
               ref_len: int | None = None, deg_len: int | None = None) -> int:
        """Queue one pair; host arrays are copied before this returns. With
        device_inputs, ref/deg are device addresses (ints) that must stay
        valid until the request completes."""
        t = c_uint64()
        if device_inputs:
            rp, dp, rl, dl = c_void_p(ref), c_void_p(deg), ref_len, deg_len
        else:
            ref = np.ascontiguousarray(ref, dtype=np.float64)
            deg = np.ascontiguousarray(deg, dtype=np.float64)
            rp, dp, rl, dl = ref.ctypes.data_as(c_void_p), deg.ctypes.data_as(c_void_p), ref.size, deg.size
        _check(lib.visqol_b200_server_submit(self._handle, mode, rp, rl, dp, dl, sample_rate,
                                             DEVICE_INPUTS if device_inputs else 0, ctypes.byref(t)))
        return t.value

    def next(self, timeout_ms: int = -1):
        """(ticket, status, result dict or None) of the next completed
        request, or None when nothing completed within timeout_ms."""
        t, st, out = c_uint64(), c_int32(), POINTER(Result)()
        rc = lib.visqol_b200_server_next(self._handle, timeout_ms, ctypes.byref(t), ctypes.byref(st),
                                         ctypes.byref(out))
        if rc == PENDING:
            return None
        _check(rc)
        res = None
        if out:
            try:
                res = result_dict(out.contents)
            finally:
                lib.visqol_result_free(out)
        return t.value, st.value, res

    def stats(self, reset: bool = False) -> dict:
        st = ServeStats()
        _check(lib.visqol_b200_server_stats(self._handle, ctypes.byref(st), int(bool(reset))))
        return {name: getattr(st, name) for name, _ in ServeStats._fields_}


class Prepared:
    """Owns a ``visqol_b200_prepared`` (see Context.prepare)."""

    def __init__(self, ctx: Context, refs, sample_rate: int, device_inputs: bool, ref_lens):
        n = len(refs)
        if device_inputs:
            rp = (c_void_p * n)(*refs)
            rl = (c_size_t * n)(*ref_lens)
        else:
            refs = [np.ascontiguousarray(r, dtype=np.float64) for r in refs]
            rp = (c_void_p * n)(*[r.ctypes.data for r in refs])
            rl = (c_size_t * n)(*[r.size for r in refs])
        handle = c_void_p()
        _check(lib.visqol_b200_prepare(ctx._handle, n, rp, rl, sample_rate, DEVICE_INPUTS if device_inputs else 0,
                                       ctypes.byref(handle)))
        self._handle = handle

    def close(self) -> None:
        if getattr(self, "_handle", None):
            lib.visqol_b200_prepared_free(self._handle)
            self._handle = None

    def __del__(self):
        self.close()


def lattice_predict(fvnsim, fvnsim10, fstdnsim, fvdegenergy, model_path: str | None = None) -> float:
    """Speech-mode TF-Lattice MOS of one set of per-band features (host only)."""
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (fvnsim, fvnsim10, fstdnsim, fvdegenergy)]
    mos = c_double()
    _check(lib.visqol_b200_lattice_predict(os.fsencode(model_path) if model_path else None, arrs[0].size,
                                           *[_dptr(a) for a in arrs], ctypes.byref(mos)))
    return mos.value


def autotune_choices() -> list[dict]:
    """Launch shapes the autotuner chose in this process."""
    n = c_size_t()
    _check(lib.visqol_b200_autotune_choices(None, 0, ctypes.byref(n)))
    rows = (c_int32 * (5 * max(1, n.value)))()
    _check(lib.visqol_b200_autotune_choices(rows, n.value, ctypes.byref(n)))
    names = {0: "gammatone_frames_per_cta", 1: "nsim_table_offsets_per_cta", 2: "lag_column_passes",
             3: "gammatone_fast_shape", 4: "gammatone_f64_staged"}
    return [{"device": rows[5 * i], "kernel": names.get(rows[5 * i + 1], str(rows[5 * i + 1])),
             "variant": (rows[5 * i + 2], rows[5 * i + 3]), "choice": rows[5 * i + 4]} for i in range(n.value)]
