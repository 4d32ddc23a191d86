"""GPU parity: cjx_slice_ctf_forward (through the C-ABI) against the float64 oracle.

Tolerance: relative L2 error per image <= 1e-5 (helpers.IMAGE_REL_L2_TOL).
"""

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import IMAGE_REL_L2_TOL, make_volume, random_specs, rel_l2_per_image, specs_to_model_args

pytestmark = pytest.mark.gpu


def _device_volume(grid):
    import torch

    from cryojax_b200 import simulator as S

    return S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())


def _run_model(grid, specs, *, transfer=True, translate=True, quantity=False, integrator_kw=None, chunk=0):
    from cryojax_b200 import simulator as S

    pose, tt, cfg = specs_to_model_args(specs)
    vol = _device_volume(grid)
    integ = S.FourierSliceExtraction(outputs_integral=quantity, **(integrator_kw or {}))
    model = S.make_image_model(vol, cfg, pose, tt if transfer else None, volume_integrator=integ,
                               applies_translation=translate, simulates_quantity=quantity)
    params = model.image_params()
    out = integ.run(vol, cfg, params, model._flags(), images_per_chunk=chunk)
    return out.cpu().numpy()


def _oracle(grid, fs, specs, **kw):
    return np.stack([O.compute_fourier_image(grid, fs, s, **kw) for s in specs])


CASES = [
    # (box, pad_scale, shape, padded_shape)  -- N = int(box * pad_scale)
    (32, 2.0, (32, 32), None),     # crop 64 -> 32 (the configs' resize)
    (32, 2.0, (64, 64), None),     # no resize: fused direct kernel
    (32, 2.0, (40, 24), None),     # non-square crop
    (32, 2.0, (70, 66), None),     # pad 64 -> 70 x 66
    (32, 2.0, (80, 48), None),     # pad y, crop x
    (31, 2.0, (31, 31), None),     # N = 62 (even), odd image
    (25, 1.0, (25, 25), None),     # odd N = 25, no resize
    (32, 1.3, (41, 41), None),     # prime N = 41: direct-DFT fallback, no resize
    (32, 1.3, (30, 30), (44, 42)), # prime N with pad and padded_shape != shape
    (48, 2.0, (48, 48), None),     # N = 96 = 2^5 * 3
    (40, 2.0, (40, 40), None),     # N = 80 = 2^4 * 5, image 40 = 2^3 * 5
    (32, 2.0, (64, 33), None),     # register column pass (Py = 64), odd Px: no x-Nyquist column
    (32, 2.0, (32, 40), None),     # register column pass, Px = 40 through the shared-memory row pass
]


@pytest.mark.parametrize("box,pad_scale,shape,padded", CASES)
def test_linear_image_model_matches_oracle(cuda_device, box, pad_scale, shape, padded):
    vol, grid, fs = make_volume(box, 60, seed=box, pad_scale=pad_scale)
    specs = random_specs(6, seed=7 * box, shape=shape, padded_shape=padded)
    got = _run_model(grid, specs)
    ref = _oracle(grid, fs, specs)
    errs = rel_l2_per_image(got, ref)
    assert max(errs) <= IMAGE_REL_L2_TOL, errs


@pytest.mark.parametrize("shape", [(32, 32), (64, 64)])
def test_integrate_only_matches_oracle(cuda_device, shape):
    """FourierSliceExtraction.integrate (no CTF, no translation), outputs_integral=True."""
    from cryojax_b200 import simulator as S

    vol, grid, fs = make_volume(32, 80, seed=3)
    specs = random_specs(4, seed=11, shape=shape)
    pose, _, cfg = specs_to_model_args(specs)
    dvol = _device_volume(grid).rotate_to_pose(pose)
    got = S.FourierSliceExtraction(outputs_integral=True).integrate(dvol, cfg).cpu().numpy()
    ref = np.stack([
        O.fourier_slice_integrate(grid, O.rotate_frequency_slice(fs, O.quat_normalize(s.wxyz)), s.padded_shape,
                                  s.pixel_size, outputs_integral=True)
        for s in specs])
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


@pytest.mark.parametrize("shape", [(32, 32), (64, 64)])
def test_envelope_offset_z_and_contrast_model(cuda_device, shape):
    vol, grid, fs = make_volume(32, 60, seed=5)
    specs = random_specs(5, seed=13, shape=shape, offset_z=True, envelope=True)
    got = _run_model(grid, specs, quantity=True)
    ref = _oracle(grid, fs, specs, outputs_integral=True, simulates_quantity=True)
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


@pytest.mark.parametrize("shape", [(32, 32), (64, 64)])
def test_projection_model_and_fill_value(cuda_device, shape):
    vol, grid, fs = make_volume(32, 60, seed=9)
    specs = random_specs(4, seed=17, shape=shape)
    fill = 0.25 - 0.5j
    got = _run_model(grid, specs, transfer=False, integrator_kw=dict(fill_value=fill))
    ref = _oracle(grid, fs, specs, apply_ctf=False, cval=fill)
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


def test_out_of_bounds_rules(cuda_device):
    """Default: negative corner indices wrap (the reference's rule); optional pure zero fill."""
    # sharp Gaussians put spectrum into the plane corners that leave the cube
    vol, grid, fs = make_volume(32, 60, seed=21, sigma_range=(0.4, 0.7))
    specs = random_specs(4, seed=23, shape=(32, 32))
    ref_wrap = _oracle(grid, fs, specs)
    ref_zero = _oracle(grid, fs, specs, wrap_negative=False)
    assert max(rel_l2_per_image(ref_wrap, ref_zero)) > 1e-3  # the two rules really differ here
    got_zero = _run_model(grid, specs, integrator_kw=dict(out_of_bounds_mode="zero_fill_negative"))
    assert max(rel_l2_per_image(got_zero, ref_zero)) <= IMAGE_REL_L2_TOL
    got_wrap = _run_model(grid, specs)
    assert max(rel_l2_per_image(got_wrap, ref_wrap)) <= IMAGE_REL_L2_TOL


@pytest.mark.parametrize("chunk", [1, 3, 0])
def test_chunking_is_invisible(cuda_device, chunk):
    vol, grid, fs = make_volume(32, 60, seed=31)
    specs = random_specs(7, seed=37, shape=(32, 32))
    got = _run_model(grid, specs, chunk=chunk)
    ref = _oracle(grid, fs, specs)
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("ilp", [1, 2, 4])
def test_processing_order_and_gather_ilp_are_invisible(cuda_device, ilp, mode):
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200 import simulator as S

    vol, grid, fs = make_volume(32, 60, seed=33)
    specs = random_specs(9, seed=39, shape=(32, 32))
    pose, tt, cfg = specs_to_model_args(specs)
    dvol = _device_volume(grid)
    model = S.make_image_model(dvol, cfg, pose, tt)
    order = S.orientation_order(pose.rotation_matrices())
    old = nat.tuning_get(nat.CJX_TUNE_GATHER_ILP), nat.tuning_get(nat.CJX_TUNE_GATHER_MODE)
    try:
        nat.tuning_set(nat.CJX_TUNE_GATHER_ILP, ilp)
        nat.tuning_set(nat.CJX_TUNE_GATHER_MODE, mode)
        got = model.volume_integrator.run(dvol, cfg, model.image_params(), model._flags(), order=order,
                                          images_per_chunk=4).cpu().numpy()
    finally:
        nat.tuning_set(nat.CJX_TUNE_GATHER_ILP, old[0])
        nat.tuning_set(nat.CJX_TUNE_GATHER_MODE, old[1])
    ref = _oracle(grid, fs, specs)
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


@pytest.mark.parametrize("box,pad_scale,shape", [(32, 2.0, (32, 32)), (31, 2.0, (31, 31)), (32, 1.3, (30, 30)),
                                                  (32, 2.0, (64, 64)), (25, 1.0, (25, 25))])
def test_linear_and_bricked_layouts_match_oracle(cuda_device, box, pad_scale, shape):
    from cryojax_b200 import simulator as S

    vol, grid, fs = make_volume(box, 60, seed=box + 3, pad_scale=pad_scale)
    specs = random_specs(4, seed=box + 5, shape=shape)
    ref = _oracle(grid, fs, specs)
    outs = {}
    for bricked, pairs in ((False, False), (True, False), (True, True)):
        got = _run_model(grid, specs, integrator_kw=dict(use_bricked_layout=bricked, pair_layout=pairs))
        assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL, (bricked, pairs)
        outs[(bricked, pairs)] = got
    # the x-pair layout reads the same values in the same order as the bricked one
    np.testing.assert_array_equal(outs[(True, True)], outs[(True, False)])


def test_brick_volume_pairs_layout(cuda_device):
    """cjx_brick_volume_pairs: entry (z, y, x) = (g(z, y, x), g(z, y, x + 1)) at the bricked address."""
    import torch

    from cryojax_b200 import _native as nat

    n = 21
    g = (np.arange(n**3, dtype=np.float32) + 1j * np.arange(n**3, dtype=np.float32)[::-1]).reshape(n, n, n)
    gt = torch.as_tensor(g.astype(np.complex64)).cuda()
    b = nat.brick_volume(gt).cpu().numpy()
    p = nat.brick_volume_pairs_new(gt).cpu().numpy()
    assert p.size == 2 * b.size
    np.testing.assert_array_equal(p[0::2], b)  # first halves: the bricked copy
    nb = (n + 7) // 8

    def addr(z, y, x):
        def spread(i):
            return (i & 1) | ((i & 2) << 2) | ((i & 4) << 4)
        blk = ((z >> 3) * nb + (y >> 3)) * nb + (x >> 3)
        return blk * 512 + spread(x & 7) + (spread(y & 7) << 1) + (spread(z & 7) << 2)

    rng = np.random.default_rng(0)
    for z, y, x in rng.integers(0, n, (50, 3)):
        e = addr(z, y, x)
        assert p[2 * e] == g[z, y, x]
        assert p[2 * e + 1] == (g[z, y, x + 1] if x + 1 < n else 0)


def test_brick_volume_layout(cuda_device):
    """cjx_brick_volume places voxel (z, y, x) at its Morton-in-block address."""
    import torch

    from cryojax_b200 import _native as nat

    n = 21
    g = (np.arange(n**3, dtype=np.float32) + 1j * np.arange(n**3, dtype=np.float32)[::-1]).reshape(n, n, n)
    b = nat.brick_volume(torch.as_tensor(g.astype(np.complex64)).cuda()).cpu().numpy()
    nb = (n + 7) // 8
    assert b.size == nb**3 * 512

    def spread(v):
        return (v & 1) | ((v & 2) << 2) | ((v & 4) << 4)

    rng = np.random.default_rng(0)
    for z, y, x in rng.integers(0, n, size=(200, 3)):
        addr = ((z // 8) * nb + (y // 8)) * nb * 512 + (x // 8) * 512 + spread(x % 8) + (spread(y % 8) << 1) + (
            spread(z % 8) << 2)
        assert b[addr] == g[z, y, x]
    # every voxel of g is nonzero; the padding of the last blocks is zero
    assert np.count_nonzero(b) == n**3


def test_simulate_real_space_matches_oracle(cuda_device):
    from cryojax_b200 import simulator as S

    vol, grid, fs = make_volume(32, 60, seed=41)
    specs = random_specs(3, seed=43, shape=(28, 28), padded_shape=(32, 32))
    pose, tt, cfg = specs_to_model_args(specs)
    model = S.make_image_model(_device_volume(grid), cfg, pose, tt)
    got = model.simulate().cpu().numpy()
    ref = np.stack([O.simulate(grid, fs, s) for s in specs])
    assert got.shape == (3, 28, 28)
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


def test_from_real_voxel_grid_matches_oracle(cuda_device):
    from cryojax_b200 import simulator as S

    vol, grid, fs = make_volume(20, 30, seed=51, pad_scale=1.3)
    dvol = S.FourierVoxelGridVolume.from_real_voxel_grid(vol, pad_scale=1.3)
    assert dvol.shape == grid.shape
    assert O.relative_l2(dvol.fourier_voxel_grid.cpu().numpy(), grid) < 1e-6


def _golden_volume():
    import json
    import os

    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    vol = np.load(os.path.join(here, "3j9g_potential_ps4_4.npy")).astype(np.float64)
    return vol, json.load(open(os.path.join(here, "3j9g_potential_ps4_4.json")))["voxel_size_A"]


def test_reference_fixture_volume_and_config(cuda_device):
    """The reference's image-model fixture: its 64^3 map at pad 1.3 (N = 83, prime), images 74^2 padded
    to 83^2, default CTF; identity and random poses; Fourier image and cropped real-space image."""
    import torch

    from cryojax_b200 import simulator as S

    vol, voxel = _golden_volume()
    grid, fs = O.fourier_voxel_grid_from_real_voxel_grid(vol, pad_scale=1.3)
    n = grid.shape[0]
    rng = np.random.default_rng(3)
    q = np.concatenate([[[1.0, 0.0, 0.0, 0.0]], O.uniform_poses(4, 5, 0.0)[0]])
    specs = [O.ImageSpec(shape=(int(0.9 * n), int(0.9 * n)), padded_shape=(n, n), pixel_size=voxel, wxyz=qq,
                         offset_in_angstroms=rng.uniform(-8, 8, 2)) for qq in q]
    pose, tt, cfg = specs_to_model_args(specs)
    V = S.FourierVoxelGridVolume.from_real_voxel_grid(torch.as_tensor(vol), pad_scale=1.3)
    model = S.make_image_model(V, cfg, pose, tt)
    got_f = model.compute_fourier_image().cpu().numpy()
    ref_f = np.stack([O.compute_fourier_image(grid, fs, s) for s in specs])
    assert max(rel_l2_per_image(got_f, ref_f)) <= IMAGE_REL_L2_TOL
    got = model.simulate().cpu().numpy()
    ref = np.stack([O.simulate(grid, fs, s) for s in specs])
    assert got.shape == (5, 74, 74)
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


@pytest.mark.parametrize("extra_y, extra_x", [(1, 1), (1, 0), (0, 1)])
def test_even_vs_odd_image_shape_on_the_device(cuda_device, extra_y, extra_x):
    """cryojax tests/test_image_model.py:83-105 through the device path (odd-N resize, N = 83)."""
    import torch

    from cryojax_b200 import simulator as S

    vol, voxel = _golden_volume()
    V = S.FourierVoxelGridVolume.from_real_voxel_grid(torch.as_tensor(vol), pad_scale=1.3)
    n = V.shape[0]
    control, test = (n, n), (n + extra_y, n + extra_x)
    pose = S.EulerAnglePose()
    tt = S.ContrastTransferTheory(S.AstigmaticCTF())
    a = S.make_image_model(V, S.BasicImageConfig(test, voxel, 300.0), pose, tt).simulate().cpu().numpy()
    b = S.make_image_model(V, S.BasicImageConfig(control, voxel, 300.0), pose, tt).simulate().cpu().numpy()
    np.testing.assert_allclose(O.crop_to_shape(a, control), b, atol=1e-4)
