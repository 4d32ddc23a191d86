"""GPU: pose/defocus refinement through the adjoint kernels, and the area downsample.

Refinement: observed images are the float64 oracle's simulations at seeded
true poses and defoci (64^2 images from a 128^3 grid, light noise at SNR
5); starting 2-4 degrees and up to
+-300 A away, 20 steps must bring the rotation within 0.5 degree of the
truth and remove at least 95 % of the loss excess over the true parameters
(start - loss at the truth; the noisy data's optimum, not the truth, is
what the descent can reach) for at least 14 of 16 images, the defocus
within 200 A for all, and no image's loss may end above its starting loss.
"""

import copy

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import make_volume, specs_to_model_args

pytestmark = pytest.mark.gpu


def _area_ref(x, h, w):
    n, H, W = x.shape

    def weights(N, m):
        f = N / m
        wt = np.zeros((m, N))
        for i in range(m):
            a0, a1 = i * f, (i + 1) * f
            for p in range(int(np.floor(a0)), min(N, int(np.ceil(a1)))):
                wt[i, p] = max(0.0, min(a1, p + 1) - max(a0, p))
        return wt / f

    return np.einsum("iy,nyx,jx->nij", weights(H, h), x, weights(W, w))


@pytest.mark.parametrize("H,h", [(320, 128), (64, 32), (100, 64)])
def test_area_downsample(cuda_device, H, h):
    import torch

    from cryojax_b200 import _native as nat

    rng = np.random.default_rng(H)
    x = rng.standard_normal((5, H, H)).astype(np.float32)
    out = torch.empty((5, h, h), dtype=torch.float32, device="cuda")
    nat.area_downsample(torch.as_tensor(x).cuda(), out)
    ref = _area_ref(x.astype(np.float64), h, h)
    assert np.abs(out.cpu().numpy() - ref).max() <= 1e-5 * np.abs(ref).max() + 1e-6


def test_refinement_converges_to_the_true_pose(cuda_device):
    import torch

    from cryojax_b200 import rotations as rot
    from cryojax_b200 import simulator as S
    from cryojax_b200.refine import refine_poses, rotation_angle_deg

    n = 16
    _, grid, fs = make_volume(64, 150, seed=3)
    q_true, _ = O.uniform_poses(n, 4, 0.0)
    rng = np.random.default_rng(5)
    specs, obs, true_df = [], [], []
    for b in range(n):
        s = O.ImageSpec(shape=(64, 64), pixel_size=2.0, wxyz=q_true[b], offset_in_angstroms=(0.0, 0.0),
                        defocus_in_angstroms=rng.uniform(8000, 15000), astigmatism_in_angstroms=100.0,
                        astigmatism_angle=20.0)
        true_df.append(s.defocus_in_angstroms)
        img = O.simulate(grid, fs, s)
        obs.append(img + rng.standard_normal(img.shape) * np.sqrt(img.var() / 5.0))
        s2 = copy.deepcopy(s)
        axis = rng.standard_normal(3)
        axis /= np.linalg.norm(axis)
        s2.wxyz = O.quat_compose(O.so3_exp(np.deg2rad(rng.uniform(2, 4)) * axis), q_true[b])
        s2.defocus_in_angstroms += rng.uniform(-300, 300)
        specs.append(s2)
    pose, tt, cfg = specs_to_model_args(specs)
    vol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
    model = S.make_image_model(vol, cfg, pose, tt)
    res = refine_poses(model, np.stack(obs), steps=20, rot_step_deg=2.0, defocus_step=150.0)
    err = rotation_angle_deg(res.rotations, rot.quat_to_matrix(q_true))
    assert np.all(res.loss <= res.loss_history[0] + 1e-9)
    assert np.sum(err < 0.5) >= 14, err
    assert np.all(np.abs(res.defocus - np.array(true_df)) < 200.0), (res.defocus, true_df)
    true_specs = []
    for b in range(n):
        t = copy.deepcopy(specs[b])
        t.wxyz, t.defocus_in_angstroms = q_true[b], true_df[b]
        true_specs.append(t)
    pose_t, tt_t, _ = specs_to_model_args(true_specs)
    at_truth = refine_poses(S.make_image_model(vol, cfg, pose_t, tt_t), np.stack(obs), steps=1).loss
    start = res.loss_history[0]
    assert np.sum(start - res.loss >= 0.95 * (start - at_truth)) >= 14, (start, res.loss, at_truth)


def test_refinement_on_a_spline_volume(cuda_device):
    """The same refinement through a FourierVoxelSplineVolume, against spline simulations of the truth."""
    import torch

    from cryojax_b200 import rotations as rot
    from cryojax_b200 import simulator as S
    from cryojax_b200.refine import refine_poses, rotation_angle_deg

    n = 8
    _, grid, fs = make_volume(64, 150, seed=6)
    coef = O.compute_spline_coefficients(grid)
    q_true, _ = O.uniform_poses(n, 7, 0.0)
    rng = np.random.default_rng(8)
    specs, obs = [], []
    for b in range(n):
        s = O.ImageSpec(shape=(64, 64), pixel_size=2.0, wxyz=q_true[b], offset_in_angstroms=(0.0, 0.0),
                        defocus_in_angstroms=rng.uniform(8000, 15000), astigmatism_in_angstroms=100.0,
                        astigmatism_angle=20.0)
        img = O.simulate(coef, fs, s, spline=True)
        obs.append(img + rng.standard_normal(img.shape) * np.sqrt(img.var() / 5.0))
        s2 = copy.deepcopy(s)
        axis = rng.standard_normal(3)
        axis /= np.linalg.norm(axis)
        s2.wxyz = O.quat_compose(O.so3_exp(np.deg2rad(rng.uniform(2, 4)) * axis), q_true[b])
        specs.append(s2)
    pose, tt, cfg = specs_to_model_args(specs)
    vol = S.FourierVoxelSplineVolume(torch.as_tensor(coef.astype(np.complex64)).cuda())
    res = refine_poses(S.make_image_model(vol, cfg, pose, tt), np.stack(obs), steps=20, rot_step_deg=2.0,
                       defocus_step=150.0)
    err = rotation_angle_deg(res.rotations, rot.quat_to_matrix(q_true))
    assert np.all(res.loss <= res.loss_history[0] + 1e-9)
    assert np.sum(err < 0.5) >= 7, err


def test_refinement_on_the_ewald_sphere(cuda_device):
    """The same refinement through EwaldSphereExtraction at 40 kV (the surface leaves the plane by up to about a
    voxel at its corners), against the oracle's Ewald contrast simulations of the truth."""
    import torch

    from cryojax_b200 import rotations as rot
    from cryojax_b200 import simulator as S
    from cryojax_b200.refine import refine_poses, rotation_angle_deg

    n = 8
    _, grid, fs = make_volume(64, 150, seed=10)
    q_true, _ = O.uniform_poses(n, 11, 0.0)
    rng = np.random.default_rng(12)
    specs, obs = [], []
    for b in range(n):
        s = O.ImageSpec(shape=(64, 64), pixel_size=2.0, voltage_in_kilovolts=40.0, wxyz=q_true[b],
                        offset_in_angstroms=(0.0, 0.0), defocus_in_angstroms=rng.uniform(8000, 15000),
                        astigmatism_in_angstroms=100.0, astigmatism_angle=20.0, amplitude_contrast_ratio=0.1)
        img = O.simulate(grid, fs, s, ewald=True)
        obs.append(img + rng.standard_normal(img.shape) * np.sqrt(img.var() / 5.0))
        s2 = copy.deepcopy(s)
        axis = rng.standard_normal(3)
        axis /= np.linalg.norm(axis)
        s2.wxyz = O.quat_compose(O.so3_exp(np.deg2rad(rng.uniform(2, 4)) * axis), q_true[b])
        specs.append(s2)
    pose, tt, cfg = specs_to_model_args(specs)
    vol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
    integ = S.EwaldSphereExtraction(outputs_integral=False)
    res = refine_poses(S.make_image_model(vol, cfg, pose, tt, volume_integrator=integ), np.stack(obs), steps=20,
                       rot_step_deg=2.0, defocus_step=150.0)
    err = rotation_angle_deg(res.rotations, rot.quat_to_matrix(q_true))
    assert np.all(res.loss <= res.loss_history[0] + 1e-9)
    assert np.sum(err < 0.5) >= 7, err
