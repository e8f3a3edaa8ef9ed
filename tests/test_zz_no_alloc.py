"""visqol_b200_dp_static (device buffers from the library's reserved array)
against visqol_b200_dp (buffers from cudaMalloc) on the same tables.

Two calls in a row on different shapes, the second smaller than the first,
so that anything the first call left in the shared array would show up in
the second's results."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(seed, np_, nfd, ties):
    rng = np.random.default_rng(seed)
    sims = rng.uniform(-0.2, 1.0, (np_, nfd))
    if ties:
        sims = np.round(sims, 1)
    idx = np.sort(rng.integers(0, nfd, np_))
    radius = int(rng.integers(1, 200))
    lo = np.maximum(0, idx - radius)
    hi = np.maximum(lo, np.minimum(idx + radius, nfd - 1))
    return sims, lo, hi


def test_static_matches_allocating_two_calls(native):
    cases = [_case(101, 40, 3000, False), _case(102, 9, 400, True)]
    got = [native.dp(*c, static_scratch=True) for c in cases]
    want = [native.dp(*c) for c in cases]
    for (goff, gval, greach), (woff, wval, wreach) in zip(got, want):
        assert greach == wreach
        assert np.array_equal(goff, woff) and np.array_equal(gval, wval)


def test_static_at_the_size_limit(native):
    sims, lo, hi = _case(103, 64, 4096, True)  # 262144 cells, the maximum
    assert native.dp(sims, lo, hi, static_scratch=True)[0].tolist() == native.dp(sims, lo, hi)[0].tolist()


def test_static_rejects_oversize(native):
    sims, lo, hi = _case(104, 65, 4096, False)  # one row past the limit
    with pytest.raises(native.NativeError) as e:
        native.dp(sims, lo, hi, static_scratch=True)
    assert e.value.code == native.E_INVALID_ARGUMENT and "static scratch" in str(e.value)
