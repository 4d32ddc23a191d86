"""HEALPix RING pixel centres and the orientation grid (CPU)."""

import numpy as np
import pytest

from cryojax_b200 import healpix as hp
from cryojax_b200 import rotations as rot


@pytest.mark.parametrize("nside", [1, 2, 4, 8])
def test_ring_structure(nside):
    theta, phi = hp.pix2ang_ring(nside)
    npix = 12 * nside * nside
    assert theta.size == npix
    z = np.round(np.cos(theta), 12)
    rings = np.unique(z)
    assert rings.size == 4 * nside - 1
    # north cap ring i has 4 i pixels, equatorial rings 4 nside
    for i in range(1, nside):
        assert np.sum(z == np.round(1 - i * i / (3.0 * nside * nside), 12)) == 4 * i
    # symmetric about the equator and in azimuth
    np.testing.assert_allclose(np.sort(z), np.sort(-z), atol=1e-12)
    assert np.all((phi >= 0) & (phi < 2 * np.pi))


def test_nside8_equal_area_and_spacing():
    d = hp.pixel_directions(8)
    assert d.shape == (768, 3)
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-12)
    # nearest-centre assignment of uniform directions is close to uniform (equal areas)
    rng = np.random.default_rng(0)
    v = rng.standard_normal((400000, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    counts = np.bincount(hp.nearest_pixel(8, v), minlength=768)
    expected = 400000 / 768
    assert np.abs(counts - expected).max() < 0.25 * expected
    # nearest-neighbour spacing about sqrt(4 pi / 768) = 7.3 degrees
    ang = np.degrees(np.arccos(np.clip(d @ d.T, -1, 1)))
    np.fill_diagonal(ang, 180)
    nn = ang.min(axis=1)
    assert 5.0 < nn.mean() < 9.0 and nn.max() < 10.0


def test_orientation_grid_normals_are_the_directions():
    g = hp.OrientationGrid(8, 48)
    assert g.size == 36864
    idx = np.array([0, 47, 48, 1000, 36863])
    R = g.rotation_matrices(idx)
    d = hp.pixel_directions(8)[idx // 48]
    np.testing.assert_allclose(R[:, :, 2], d, atol=1e-12)
    assert np.all(g.direction_of(R) == idx // 48)
    # in-plane steps of 7.5 degrees rotate the plane about its normal
    R0, R1 = g.rotation_matrices([48 * 5]), g.rotation_matrices([48 * 5 + 1])
    c = np.clip(np.dot(R0[0][:, 0], R1[0][:, 0]), -1, 1)
    assert abs(np.degrees(np.arccos(c)) - 7.5) < 1e-9
