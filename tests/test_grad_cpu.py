"""The host half of the gradient (no GPU): each reverse step against central
differences of the oracle's forward function, with random weights on its
outputs (a scalar loss L = sum w * output)."""

import numpy as np
import pytest


def central(f, x, idx, h):
    xp, xm = x.copy(), x.copy()
    xp[idx] += h
    xm[idx] -= h
    return (f(xp) - f(xm)) / (2 * h)


@pytest.mark.parametrize("ncols", [30, 27, 2])
def test_patch_similarity_grad(native, oracle, ncols):
    """measurePatchSimilarity's reverse: band means, standard deviations and
    deg energies weighted by random gradients, against central differences
    over ref and deg cells (prepared-spectrogram values, dB above a floor)."""
    rng = np.random.default_rng(ncols)
    nb = 32
    ref = rng.uniform(5.0, 40.0, (nb, ncols))
    deg = ref + rng.normal(0.0, 3.0, (nb, ncols))
    wm, ws, we = rng.standard_normal(nb), rng.standard_normal(nb), rng.standard_normal(nb)

    def loss(r, d):
        _, m, s, e = oracle.patch_similarity(r, d)
        return float(np.dot(wm, m) + np.dot(ws, s) + np.dot(we, e))

    dref, ddeg = native.patch_similarity_grad(ref, deg, wm, ws, we)
    for _ in range(40):
        idx = (int(rng.integers(nb)), int(rng.integers(ncols)))
        gd = central(lambda d: loss(ref, d), deg, idx, 1e-5)
        gr = central(lambda r: loss(r, deg), ref, idx, 1e-5)
        assert abs(ddeg[idx] - gd) <= 1e-6 * max(1.0, abs(gd)), (idx, ddeg[idx], gd)
        assert abs(dref[idx] - gr) <= 1e-6 * max(1.0, abs(gr)), (idx, dref[idx], gr)


def test_prepare_grad(native, oracle):
    """prepareForComparison's reverse through the dB conversion, the per-frame
    floors (floored cells pass their gradient to the cell that set the
    floor) and the joint minimum (every cell's gradient flows, negated, to
    the minimum's cell), against central differences over raw degraded
    cells, with some frames quiet enough to be floored."""
    rng = np.random.default_rng(5)
    nb, nfr, nfd = 32, 40, 44
    ref = np.exp(rng.uniform(-6, 0, (nb, nfr)))
    deg = np.exp(rng.uniform(-6, 0, (nb, nfd)))
    deg[:, 10] *= 1e-4  # a quiet frame: floored cells
    deg[3, 20] *= 1e-8  # a deep cell: the joint minimum
    gr, gd = rng.standard_normal((nb, nfr)), rng.standard_normal((nb, nfd))

    def loss(d):
        pr, pd = oracle.prepare_for_comparison(ref, d)
        return float(np.sum(gr * pr) + np.sum(gd * pd))

    got = native.prepare_grad(ref, deg, gr, gd)
    cells = [(3, 20), (0, 10), (31, 10)] + [(int(rng.integers(nb)), int(rng.integers(nfd))) for _ in range(40)]
    for idx in cells:
        want = central(loss, deg, idx, 1e-4 * deg[idx])
        assert abs(got[idx] - want) <= 1e-5 * max(1.0, abs(want)), (idx, got[idx], want)
