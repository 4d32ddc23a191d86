"""GPU parity: FourierVoxelSplineVolume -- cubic-spline coefficients
(cjx_spline_coefficients) and cubic-spline slice extraction (CJX_GRID_SPLINE)
through the C-ABI, against the float64 oracle.

Tolerances: coefficients within 1e-6 of the oracle's largest magnitude
(complex64 storage of a double-precision solve); images within relative L2
error IMAGE_REL_L2_TOL (1e-5) per image, as for the trilinear path; the
C-order and bricked coefficient layouts agree to 1e-6; search scores within
the NCC tolerance of the plain search tests (5e-5).
"""

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import IMAGE_REL_L2_TOL, make_volume, random_specs, rel_l2_per_image, specs_to_model_args

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(4, 4, 4), (16, 16, 16), (33, 33, 33), (64, 64, 64)])
def test_coefficients_match_oracle(cuda_device, shape):
    import torch

    from cryojax_b200 import _native as nat

    rng = np.random.default_rng(shape[0])
    g = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    got = nat.spline_coefficients(torch.as_tensor(g).cuda()).cpu().numpy()
    ref = O.compute_spline_coefficients(g.astype(np.complex128))
    assert got.shape == ref.shape == tuple(s + 2 for s in shape)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err <= 1e-6, err


def test_coefficients_reproduce_a_large_grid(cuda_device):
    """N = 512 (the benchmark's volume side): the [1, 4, 1] stencil of the coefficients along all three axes
    gives back the grid (the interpolation condition), checked in float64 on the device."""
    import torch

    from cryojax_b200 import _native as nat

    n = 512
    gen = torch.Generator(device="cuda").manual_seed(5)
    g = torch.randn((n, n, n), dtype=torch.complex64, device="cuda", generator=gen)
    c = nat.spline_coefficients(g)
    assert tuple(c.shape) == (n + 2,) * 3
    for z0 in (0, 255, n - 4):  # slabs of 4 output planes
        cs = c[z0:z0 + 6].to(torch.complex128)
        r = cs[:-2] + 4 * cs[1:-1] + cs[2:]
        r = r[:, :-2] + 4 * r[:, 1:-1] + r[:, 2:]
        r = r[:, :, :-2] + 4 * r[:, :, 1:-1] + r[:, :, 2:]
        err = (r - g[z0:z0 + 4].to(torch.complex128)).abs().max().item()
        assert err <= 2e-5 * g.abs().max().item(), (z0, err)


def _spline_volume(grid):
    import torch

    from cryojax_b200 import simulator as S

    return S.FourierVoxelSplineVolume.from_fourier_voxel_grid(
        S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda()))


LAYOUTS = ["linear", "bricked", "pairs"]


def _run(vol, specs, layout, chunk=0, fill=0.0):
    from cryojax_b200 import simulator as S

    pose, tt, cfg = specs_to_model_args(specs)
    integ = S.FourierSliceExtraction(outputs_integral=False, use_bricked_layout=layout != "linear",
                                     pair_layout=layout == "pairs", fill_value=fill)
    model = S.make_image_model(vol, cfg, pose, tt, volume_integrator=integ)
    return integ.run(vol, cfg, model.image_params(), model._flags(), images_per_chunk=chunk).cpu().numpy()


CASES = [
    (32, 2.0, (32, 32), None),      # crop 64 -> 32 (resize path)
    (32, 2.0, (64, 64), None),      # no resize: direct kernel
    (32, 2.0, (70, 66), None),      # pad
    (25, 1.0, (25, 25), None),      # odd N = 25, no resize
    (32, 1.3, (30, 30), (44, 42)),  # prime N = 41 with pad and padded_shape != shape
]


@pytest.mark.parametrize("box,pad_scale,shape,padded", CASES)
@pytest.mark.parametrize("layout", LAYOUTS)
def test_spline_image_model_matches_oracle(cuda_device, box, pad_scale, shape, padded, layout):
    _, grid, fs = make_volume(box, 60, seed=box, pad_scale=pad_scale)
    specs = random_specs(5, seed=3 * box, shape=shape, padded_shape=padded)
    vol = _spline_volume(grid)
    got = _run(vol, specs, layout)
    coef = O.compute_spline_coefficients(grid)
    ref = np.stack([O.compute_fourier_image(coef, fs, s, spline=True) for s in specs])
    errs = rel_l2_per_image(got, ref)
    assert max(errs) <= IMAGE_REL_L2_TOL, errs
    # and the spline image differs from the trilinear one (the flag really switched the sampler)
    lin = np.stack([O.compute_fourier_image(grid, fs, s) for s in specs])
    assert min(rel_l2_per_image(lin, ref)) > 1e-4


def test_spline_fill_value_and_faces(cuda_device):
    """Sharp features push spectrum into the plane corners that leave the cube: taps outside the
    coefficient array read the fill value (negative indices wrap once on side N + 2)."""
    _, grid, fs = make_volume(32, 60, seed=21, sigma_range=(0.4, 0.7))
    specs = random_specs(4, seed=23, shape=(32, 32))
    coef = O.compute_spline_coefficients(grid)
    fill = 0.25 - 0.5j
    vol = _spline_volume(grid)
    for layout in LAYOUTS:
        got = _run(vol, specs, layout, fill=fill)
        ref = np.stack([O.compute_fourier_image(coef, fs, s, spline=True, cval=fill) for s in specs])
        assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


def test_from_real_voxel_grid_and_reference_fixture(cuda_device):
    """FourierVoxelSplineVolume.from_real_voxel_grid on the reference's 64^3 test map at pad 1.3
    (N = 83): coefficients and images against the oracle."""
    import json
    import os

    import torch

    from cryojax_b200 import simulator as S

    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    vol = np.load(os.path.join(here, "3j9g_potential_ps4_4.npy")).astype(np.float64)
    voxel = json.load(open(os.path.join(here, "3j9g_potential_ps4_4.json")))["voxel_size_A"]
    grid, fs = O.fourier_voxel_grid_from_real_voxel_grid(vol, pad_scale=1.3)
    coef = O.compute_spline_coefficients(grid)
    V = S.FourierVoxelSplineVolume.from_real_voxel_grid(torch.as_tensor(vol), pad_scale=1.3)
    assert V.shape == grid.shape
    got_c = V.spline_coefficients.cpu().numpy()
    assert np.abs(got_c - coef).max() <= 1e-6 * np.abs(coef).max()
    n = grid.shape[0]
    rng = np.random.default_rng(3)
    q = np.concatenate([[[1.0, 0.0, 0.0, 0.0]], O.uniform_poses(4, 5, 0.0)[0]])
    specs = [O.ImageSpec(shape=(int(0.9 * n), int(0.9 * n)), padded_shape=(n, n), pixel_size=voxel, wxyz=qq,
                         offset_in_angstroms=rng.uniform(-8, 8, 2)) for qq in q]
    pose, tt, cfg = specs_to_model_args(specs)
    model = S.make_image_model(V, cfg, pose, tt)
    got = model.simulate().cpu().numpy()
    ref = np.stack([O.simulate(coef, fs, s, spline=True) for s in specs])
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


def test_multi_equals_forward(cuda_device):
    import torch

    from cryojax_b200 import _native as nat

    _, grid, fs = make_volume(32, 60, seed=4)
    vol = _spline_volume(grid)
    specs = random_specs(6, seed=8, shape=(32, 32))
    ref = _run(vol, specs, "linear")
    np.testing.assert_array_equal(_run(vol, specs, "bricked"), ref)  # same taps, same order of sums
    np.testing.assert_array_equal(_run(vol, specs, "pairs"), ref)
    from cryojax_b200 import simulator as S

    pose, tt, cfg = specs_to_model_args(specs)
    integ = S.FourierSliceExtraction(outputs_integral=False, use_bricked_layout=False)
    model = S.make_image_model(vol, cfg, pose, tt, volume_integrator=integ)
    pd = torch.as_tensor(model.image_params(), device="cuda")
    desc = nat.make_desc(64, 32, 32, model._flags() | nat.CJX_GRID_SPLINE)
    out = torch.empty((6, 32, 17), dtype=torch.complex64, device="cuda")
    ws = torch.empty(nat.workspace_size(desc, 6), dtype=torch.uint8, device="cuda")
    arr = nat.make_groups([{"desc": desc, "grid": vol.spline_coefficients, "params": pd, "out": out, "n_images": 6,
                            "workspace": ws}])
    nat.slice_ctf_forward_multi(arr, ws)
    np.testing.assert_array_equal(out.cpu().numpy(), ref)


def test_exhaustive_search_on_a_spline_volume(cuda_device):
    from cryojax_b200 import simulator as S
    from cryojax_b200.healpix import OrientationGrid
    from cryojax_b200.search import PoseSearch

    og = OrientationGrid(nside=1, n_inplane=8)  # 96 orientations
    quats = og.quaternions()
    _, grid, fs = make_volume(32, 40, seed=33)
    coef = O.compute_spline_coefficients(grid)
    rng = np.random.default_rng(32)
    true_idx = rng.choice(og.size, 3, replace=False)
    specs = [O.ImageSpec(shape=(32, 32), pixel_size=2.0, wxyz=quats[k], offset_in_angstroms=rng.uniform(-4, 4, 2),
                         defocus_in_angstroms=rng.uniform(8000, 20000)) for k in true_idx]
    obs = np.stack([O.simulate(coef, fs, s, spline=True) for s in specs])
    ref_best, ref_scores = O.grid_search_orientations(coef, fs, specs, obs, quats, spline=True)
    pose, tt, cfg = specs_to_model_args(specs)
    model = S.make_image_model(_spline_volume(grid), cfg, pose, tt)
    res = PoseSearch(og.rotation_matrices()).run(model, obs, return_scores=True)
    got = res.scores.cpu().numpy()
    assert np.abs(got - ref_scores).max() <= 5e-5
    np.testing.assert_array_equal(res.best_orientation, true_idx)
    np.testing.assert_array_equal(ref_best, true_idx)
