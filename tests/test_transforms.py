"""Filters, masks and grids (CPU): the reference's closed forms at known points.

cryojax/ndimage/transforms/_filters.py:193-226 (raised-cosine low-pass as a
fraction of Nyquist), _masks.py:321-403 (circular and square cosine masks),
cryojax/coordinates/_make_coordinate_grids.py (coordinates (i - n//2) dx,
rfft frequencies).
"""

import numpy as np

from cryojax_b200 import transforms as T
from oracle import cryojax_oracle as O


def test_grids_match_the_oracle():
    np.testing.assert_allclose(T.make_frequency_grid((10, 8), 1.5), O.make_frequency_grid((10, 8), 1.5))
    g = T.make_coordinate_grid((5, 4), 2.0)
    assert g.shape == (5, 4, 2)
    np.testing.assert_allclose(g[0, :, 0], [-4.0, -2.0, 0.0, 2.0])
    np.testing.assert_allclose(g[:, 0, 1], [-4.0, -2.0, 0.0, 2.0, 4.0])


def test_lowpass_and_highpass_filters():
    k = np.array([0.0, 0.2, 0.475, 0.4875, 0.5, 0.6])[:, None] * np.array([1.0, 0.0])  # along kx, pixel 1
    lp = T.LowpassFilter(k, 1.0, 0.95, 0.05).get()  # cutoff 0.475, rolloff 0.025 (fractions of 0.5)
    np.testing.assert_allclose(lp, [1.0, 1.0, 1.0, 0.5, 0.0, 0.0], atol=1e-12)
    hp = T.HighpassFilter(k, 1.0, 0.95, 0.05).get()
    np.testing.assert_allclose(hp, 1.0 - lp)


def test_masks():
    g = T.make_coordinate_grid((21, 21), 1.0)
    m = T.CircularCosineMask(g, radius=5.0, rolloff_width=2.0).get()
    assert m[10, 10] == 1.0 and m[10, 15] == 1.0 and m[10, 16] == 0.5 and m[10, 17] == 0.0 and m[0, 0] == 0.0
    off = T.CircularCosineMask(g, 5.0, 2.0, xy_offset=(3.0, 0.0)).get()
    assert off[10, 13] == 1.0 and off[10, 19] == 0.5
    sq = T.SquareCosineMask(g, side_length=8.0, rolloff_width=2.0).get()
    # |x| = s/2 + w exactly lies in the outer square but in neither edge band: the reference's formula
    # then takes the y edge value (1 on the axis); beyond it the mask is 0
    assert sq[10, 14] == 1.0 and sq[10, 15] == 0.5 and sq[10, 16] == 1.0 and sq[10, 17] == 0.0
    np.testing.assert_allclose(sq[15, 15], 0.25)  # both edges: product
    img = np.ones((21, 21))
    np.testing.assert_array_equal(T.CircularCosineMask(g, 5.0, 2.0)(img), m)
