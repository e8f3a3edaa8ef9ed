"""The speech-mode TF-Lattice MOS mapping (host only, no GPU): the library's
C++ interpreter against the numpy restatement in oracle/lattice.py, and the
reference's own check that a perfect match maps high
(src/lattice.zig:74-83)."""

import numpy as np
import pytest


@pytest.fixture(scope="module")
def restated():
    from oracle.lattice import Lattice
    return Lattice()


def test_perfect_match_maps_high(native):
    ones, zeros, energy = np.ones(21), np.zeros(21), np.full(21, 50.0)
    mos = native.lattice_predict(ones, ones, zeros, energy)
    assert 4.0 < mos <= 5.5


@pytest.mark.parametrize("seed", range(16))
def test_matches_restatement(native, restated, seed):
    rng = np.random.default_rng(seed)
    feats = [rng.uniform(0.3, 1.0, 21), rng.uniform(0.2, 1.0, 21), rng.uniform(0.0, 0.3, 21),
             rng.uniform(5.0, 90.0, 21)]
    got = native.lattice_predict(*feats)
    want = restated.predict(*feats)
    # f32 model, the same operations in the same order (sequential FMA dot
    # products, each rounded once): the same bits
    assert got == want, (got, want)


def test_explicit_model_path_and_errors(native, tmp_path):
    from oracle.lattice import DEFAULT_MODEL
    ones, zeros, energy = np.ones(21), np.zeros(21), np.full(21, 50.0)
    assert native.lattice_predict(ones, ones, zeros, energy, model_path=str(DEFAULT_MODEL)) == \
        native.lattice_predict(ones, ones, zeros, energy)
    with pytest.raises(native.NativeError) as e:
        native.lattice_predict(ones, ones, zeros, energy, model_path=str(tmp_path / "missing.tflite"))
    assert e.value.code == native.E_IO
    bad = tmp_path / "truncated.tflite"
    bad.write_bytes(DEFAULT_MODEL.read_bytes()[:4096])
    with pytest.raises(native.NativeError) as e:
        native.lattice_predict(ones, ones, zeros, energy, model_path=str(bad))
    assert e.value.code == native.E_MODEL
