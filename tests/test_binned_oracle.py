"""The oracle's binned pixelated detector (a numeric-angle crop the reference does not offer; its rule is this
library's own, so these are its defining properties rather than pins): per-axis overlap weights of interior pixels
sum to 1, the window's total is the area it covers, and a pattern that is constant inside the window stays
constant."""

import numpy as np

from oracle import simk_oracle as O


def test_weights_partition_interior_pixels():
    samp, outer, nb = 0.604, 60.0, 128
    w = O.binned_weights(768, samp, nb, outer)
    al = O.angles(768, samp)
    inside = np.abs(al) < outer - samp
    assert np.allclose(w[:, inside].sum(axis=0), 1.0, atol=1e-12)
    assert np.all(w[:, np.abs(al) > outer + samp] == 0)
    # each bin's weights add up to its width in pixels
    assert np.allclose(w.sum(axis=1), (2 * outer / nb) / samp, atol=1e-12)


def test_conserves_intensity_and_constants():
    g = O.Grid(96, 80, 30.0, 25.0)
    energy = 300e3
    a = O.angular_sampling(g, energy)
    outer = 0.4 * min(48 * a[0], 40 * a[1])
    p = np.ones((96, 80))
    b = O.binned_detect(p, g, energy, 16, 12, outer)
    assert np.allclose(b, b[0, 0], rtol=1e-12)  # a constant pattern stays constant
    assert abs(b.sum() - (2 * outer / a[0]) * (2 * outer / a[1])) <= 1e-9 * b.sum()
    rng = np.random.default_rng(0)
    q = rng.uniform(0, 1, (96, 80))
    al_x, al_y = O.angles(96, a[0]), O.angles(80, a[1])
    mx = np.abs(al_x) < outer - a[0]
    my = np.abs(al_y) < outer - a[1]
    q_in = q * mx[:, None] * my[None, :]  # zero outside a margin inside the window
    assert abs(O.binned_detect(q_in, g, energy, 16, 12, outer).sum() - q_in.sum()) <= 1e-12 * q_in.sum()
