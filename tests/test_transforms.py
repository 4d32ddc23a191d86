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


def test_cylinder_rectangle_and_box_masks():
    g = T.make_coordinate_grid((21, 21), 1.0)
    band = T.Cylindrical2DCosineMask(g, radius=3.0, rolloff_width=2.0).get()
    # a horizontal band |y| < 3 (x free), raised-cosine edge to |y| = 5
    assert band[10, 0] == 1.0 and band[10 + 4, 5] == 0.5 and band[10 + 5, 5] == 0.0
    rot = T.Cylindrical2DCosineMask(g, radius=3.0, rolloff_width=2.0, in_plane_rotation_angle=90.0).get()
    np.testing.assert_allclose(rot, band.T, atol=1e-12)  # rotated by 90 degrees: a vertical band
    rect = T.Rectangular2DCosineMask(g, x_width=10.0, y_width=4.0, rolloff_width=2.0).get()
    assert rect[10, 15] == 1.0 and rect[10, 16] == 0.5 and rect[12, 10] == 1.0 and rect[13, 10] == 0.5
    np.testing.assert_allclose(rect[13, 16], 0.25)
    g3 = T.make_coordinate_grid((9, 11, 13), 1.0)
    assert g3.shape == (9, 11, 13, 3) and g3[0, 0, 0].tolist() == [-6.0, -5.0, -4.0]
    box = T.Rectangular3DCosineMask(g3, 6.0, 4.0, 2.0, 2.0).get()
    assert box[4, 5, 6] == 1.0 and box[4, 5, 10] == 0.5  # x = 4: halfway through the x edge
    np.testing.assert_allclose(box[6, 8, 10], 0.125)  # three edges at their midpoints
    sph = T.SphericalCosineMask(g3, 3.0, 2.0).get()
    assert sph[4, 5, 6] == 1.0 and sph[4, 5, 10] == 0.5
    inv = T.InverseSincMask(g).get()
    np.testing.assert_allclose(inv[10, 10], 1.0)
    np.testing.assert_allclose(inv[10, 15], 1.0 / np.sinc(5 / 21))


def test_whitening_filter():
    rng = np.random.default_rng(0)
    white = rng.standard_normal((64, 48, 48)) * 3.0
    f = T.WhiteningFilter(white).get()
    assert f.shape == (48, 25) and f[0, 0] == 0.0 and f[24, 24] == 0.0
    inner = f[1:20, 1:20]
    np.testing.assert_allclose(inner.mean(), 1 / 3.0, rtol=0.03)  # white noise of std 3: flat 1/3
    sq = T.WhiteningFilter(white, outputs_squared=True).get()
    np.testing.assert_allclose(sq[1:20, 1:20].mean(), 1 / 9.0, rtol=0.05)
    # a coloured spectrum: the filter whitens it (a gentle one: the right-closed bins attribute each ring's
    # mean power to its outer edge, which under-whitens steep spectra by about slope x half a bin)
    k = np.linalg.norm(T.make_frequency_grid((48, 48)), axis=-1)
    amp = np.exp(-4 * k**2)
    noise = np.fft.irfftn(np.fft.rfftn(rng.standard_normal((64, 48, 48)), axes=(1, 2)) * amp, s=(48, 48),
                          axes=(1, 2))
    wf = T.WhiteningFilter(noise).get()
    whitened = np.fft.rfftn(noise, axes=(1, 2)) * wf
    p = (np.abs(whitened) ** 2).mean(axis=0)
    ring = lambda r0: p[(k > r0) & (k < r0 + 0.05)].mean()
    assert abs(ring(0.05) / ring(0.25) - 1.0) < 0.1
    resized = T.WhiteningFilter(white, shape=(32, 32)).get()
    assert resized.shape == (32, 17) and resized[0, 0] == 0.0
    nearest = T.WhiteningFilter(white, interpolation_mode="nearest").get()
    assert abs(nearest[1:20, 1:20].mean() * 3.0 - 1.0) < 0.03
