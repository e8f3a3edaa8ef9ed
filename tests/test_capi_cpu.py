"""The C-ABI library on a machine without a GPU: it loads, exports every
symbol the headers declare, keeps the reference's option defaults and
error codes, and refuses (never falls back) when there is no device."""

import ctypes
import os
import re
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names.update(re.findall(r"\b(visqol_\w+)\s*\(", text))
    return names


def exported_symbols(path: Path) -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", str(path)], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_exports_every_declared_symbol(native):
    decl = declared_functions()
    assert "visqol_measure_batch" in decl and "visqol_b200_measure_batch" in decl
    exported = exported_symbols(native.LIB_PATH)
    assert decl <= exported, sorted(decl - exported)
    assert set(native.EXPORTS) == decl


def test_abi_and_defaults(native):
    assert native.lib.visqol_abi_version() == 1
    o = native.Options()
    native.lib.visqol_options_default(ctypes.byref(o))
    assert (o.mode, o.search_window_radius, o.use_lattice_model, o.backend, o.precision) == (0, 60, 1, 2, 3)
    assert o.model_path is None


def test_create_argument_errors(native):
    with pytest.raises(native.NativeError) as e:
        native.Context(mode=7)
    assert e.value.code == native.E_INVALID_ARGUMENT
    with pytest.raises(native.NativeError) as e:
        native.Context(backend="cpu")
    assert e.value.code == native.E_BACKEND and "cuda" in str(e.value)
    with pytest.raises(ValueError):
        native.Context(precision="half")


@pytest.mark.skipif(bool(os.environ.get("CUDA_VISIBLE_DEVICES_FORCE")), reason="forced device")
def test_no_device_refuses_without_fallback(native):
    if native.available_backends():
        pytest.skip("a CUDA device is present")
    with pytest.raises(native.NativeError) as e:
        native.Context()
    assert e.value.code == native.E_BACKEND


@pytest.mark.skipif(bool(os.environ.get("CUDA_VISIBLE_DEVICES_FORCE")), reason="forced device")
def test_server_needs_a_device(native):
    if native.available_backends():
        pytest.skip("a CUDA device is present")
    with pytest.raises(native.NativeError) as e:
        native.Server(precision="fast")
    assert e.value.code == native.E_BACKEND


def test_server_argument_errors(native):
    o = native.Options()
    native.lib.visqol_options_default(ctypes.byref(o))
    o.backend = 0
    h = ctypes.c_void_p()
    assert native.lib.visqol_b200_server_create(ctypes.byref(o), None, ctypes.byref(h)) == native.E_BACKEND
    assert native.lib.visqol_b200_server_create(None, None, None) == native.E_INVALID_ARGUMENT
    t = ctypes.c_uint64()
    assert native.lib.visqol_b200_server_submit(None, 0, None, 0, None, 0, 48000, 0, ctypes.byref(t)) == \
        native.E_INVALID_ARGUMENT


def test_speech_lattice_is_reported(native):
    with pytest.raises(native.NativeError) as e:
        native.Context(mode=native.MODE_SPEECH, use_lattice_model=True)
    assert e.value.code in (native.E_MODEL, native.E_BACKEND)


# The reference's src/python directory, when a checkout is at hand.
REFERENCE_PY = Path(os.environ.get("VISQOL_REFERENCE_PYTHON", "/nonexistent"))


@pytest.mark.skipif(not (REFERENCE_PY / "visqol" / "_native.py").is_file(),
                    reason="VISQOL_REFERENCE_PYTHON does not name the reference's src/python")
def test_reference_python_package_loads_this_library(native):
    """The reference's own binding (src/python/visqol/_native.py) loads
    libvisqol.so through VISQOL_LIBRARY unchanged."""
    code = (
        "import visqol, visqol._native as n\n"
        "assert n.lib.visqol_abi_version() == 1\n"
        "print('backends', n.available_backends())\n"
        "try:\n"
        "    n.Context(mode=0, search_window_radius=60, use_unscaled_speech_mos_mapping=False,"
        " disable_global_alignment=False, disable_realignment=False, use_lattice_model=False,"
        " model_path=None, backend='cuda')\n"
        "    print('created')\n"
        "except n.NativeError as e:\n"
        "    print('code', e.code)\n"
    )
    env = dict(os.environ, VISQOL_LIBRARY=str(native.LIB_PATH), PYTHONPATH=str(REFERENCE_PY))
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    assert "backends" in out.stdout
    if "created" not in out.stdout:
        assert "code -6" in out.stdout
