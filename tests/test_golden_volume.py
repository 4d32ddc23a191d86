"""CPU: the oracle on the reference's own test volume (tests/golden/, from
cryojax tests/data/3j9g_potential_ps4_4.mrc, 64^3 at 4.4 A).

* even/odd image shapes: cryojax tests/test_image_model.py:83-105 restated
  exactly -- the fixture volume at pad_scale 1.3 (N = 83), identity
  EulerAnglePose, default AstigmaticCTF, shapes (N + dy, N + dx) cropped to
  (N, N) against the (N, N) image, atol = 1e-4;
* the Fourier-slice theorem at identity pose on this map
  (cryojax tests/test_volume_integrators.py:188-251, restated on the fixture).
"""

import json
import os

import numpy as np
import pytest

from oracle import cryojax_oracle as O

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixture_volume():
    vol = np.load(os.path.join(HERE, "3j9g_potential_ps4_4.npy")).astype(np.float64)
    meta = json.load(open(os.path.join(HERE, "3j9g_potential_ps4_4.json")))
    return vol, meta["voxel_size_A"]


def test_fixture_loads():
    vol, voxel = fixture_volume()
    assert vol.shape == (64, 64, 64)
    assert abs(voxel - 4.4) < 1e-6
    assert vol.max() > 0


@pytest.mark.parametrize("extra_y, extra_x", [(1, 1), (1, 0), (0, 1)])
def test_even_vs_odd_image_shape_on_the_reference_volume(extra_y, extra_x):
    vol, voxel = fixture_volume()
    grid, fs = O.fourier_voxel_grid_from_real_voxel_grid(vol, pad_scale=1.3)
    n = grid.shape[0]
    assert n == 83
    control, test = (n, n), (n + extra_y, n + extra_x)
    b = O.simulate(grid, fs, O.ImageSpec(shape=control, pixel_size=voxel))
    a = O.simulate(grid, fs, O.ImageSpec(shape=test, pixel_size=voxel))
    np.testing.assert_allclose(O.crop_to_shape(a, control), b, atol=1e-4)


def test_slice_theorem_on_the_reference_volume():
    vol, _ = fixture_volume()
    grid, fs = O.fourier_voxel_grid_from_real_voxel_grid(vol, pad_scale=1.3)
    n = grid.shape[0]
    sl = O.extract_slice(grid, O.rotate_frequency_slice(fs, np.array([1.0, 0.0, 0.0, 0.0])))
    ref = O.rfftn(O.pad_to_shape(vol, (n, n, n)).sum(axis=0))
    np.testing.assert_allclose(sl, ref, atol=1e-12 * np.abs(ref).max())
