"""GPU: squared-residual loss and gradients on the Ewald sphere against float64 central differences of the oracle.

EwaldSphereExtraction with ContrastTransferTheory's non-projection contrast
(cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:225-516,
cryojax/simulator/_transfer_theory/transfer_theory.py:100-111): the loss is
the real-space squared residual of the contrast image, as for the slice.
Each observed image is the oracle's Ewald simulation at a seeded true pose
plus white noise; the loss is evaluated at a perturbed pose (<= 3 deg,
+-2 A, +-300 A defocus).  Low accelerating voltages (20-60 kV) curve the
surface by up to a voxel, so the rotation's third column carries weight in
the pose gradient.  Central differences and tolerances as for the slice:
step 2e-7 on the quaternion, 1e-4 on offsets and defocus; loss rel 1e-5;
each gradient group rel L2 1e-4; grid-gradient entries within 1e-4 of their
own magnitude and of the largest.
"""

import copy

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import make_volume, specs_to_model_args

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4
# the full surface has twice the slice's samples, so a 1e-6 quaternion step moves one across a voxel-cell
# boundary (a kink of trilinear interpolation) more often; 2e-7 keeps the central differences on one side
QUAT_STEP = 2e-7


def _loss(grid, fs, specs, obs, spline=False):
    return sum(float(np.sum((O.simulate(grid, fs, s, ewald=True, spline=spline) - o) ** 2))
               for s, o in zip(specs, obs))


def _setup(box, shape, n, seed, kv, spline=False):
    rng = np.random.default_rng(seed)
    _, grid, fs = make_volume(box, 60, seed=seed)
    og = O.compute_spline_coefficients(grid) if spline else grid
    true_q, off = O.uniform_poses(n, seed + 1, 8.0)
    specs, obs = [], []
    for b in range(n):
        s_true = O.ImageSpec(shape=shape, pixel_size=2.0, voltage_in_kilovolts=kv, wxyz=true_q[b],
                             offset_in_angstroms=off[b], defocus_in_angstroms=rng.uniform(8000, 15000),
                             astigmatism_in_angstroms=150.0, astigmatism_angle=30.0,
                             amplitude_contrast_ratio=rng.uniform(0.05, 0.2), phase_shift=rng.uniform(0, 20))
        img = O.simulate(og, fs, s_true, ewald=True, spline=spline)
        obs.append(img + rng.standard_normal(img.shape) * np.sqrt(img.var() / 0.1))
        axis = rng.standard_normal(3)
        axis /= np.linalg.norm(axis)
        s = copy.deepcopy(s_true)
        s.wxyz = O.quat_compose(O.so3_exp(np.deg2rad(rng.uniform(0.5, 3.0)) * axis), true_q[b])
        s.offset_in_angstroms = off[b] + rng.uniform(-2, 2, 2)
        s.defocus_in_angstroms = s_true.defocus_in_angstroms + rng.uniform(-300, 300)
        specs.append(s)
    return grid, og, fs, specs, np.stack(obs)


def _model(grid, specs, layout="pairs", spline=False):
    import torch

    from cryojax_b200 import simulator as S

    pose, tt, cfg = specs_to_model_args(specs)
    vol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
    if spline:
        vol = S.FourierVoxelSplineVolume.from_fourier_voxel_grid(vol)
    integ = S.EwaldSphereExtraction(use_bricked_layout=layout != "linear", pair_layout=layout == "pairs",
                                    outputs_integral=False)  # the oracle's default
    return S.make_image_model(vol, cfg, pose, tt, volume_integrator=integ)


def _fd(f, h):
    return (f(h) - f(-h)) / (2 * h)


def _check_parameter_gradients(res, og, fs, specs, obs, spline):
    for b, s in enumerate(specs):
        ref_loss = _loss(og, fs, [s], obs[b:b + 1], spline)
        assert abs(res["loss"][b] - ref_loss) <= 1e-5 * ref_loss, (b, res["loss"][b], ref_loss)

        def with_(fn, h):
            s2 = copy.deepcopy(s)
            fn(s2, h)
            return _loss(og, fs, [s2], obs[b:b + 1], spline)

        g_fd = []
        for c in range(4):
            def fq(s2, h, c=c):
                s2.wxyz = s.wxyz + h * np.eye(4)[c]
            g_fd.append(_fd(lambda h: with_(fq, h), QUAT_STEP))
        g_fd += [_fd(lambda h: with_(lambda s2, h: setattr(s2, "offset_in_angstroms",
                                                           s.offset_in_angstroms + [h, 0]), h), 1e-4),
                 _fd(lambda h: with_(lambda s2, h: setattr(s2, "offset_in_angstroms",
                                                           s.offset_in_angstroms + [0, h]), h), 1e-4),
                 _fd(lambda h: with_(lambda s2, h: setattr(s2, "defocus_in_angstroms",
                                                           s.defocus_in_angstroms + h), h), 1e-4)]
        g_fd = np.array(g_fd)
        g_gpu = np.concatenate([res["d_wxyz"][b], res["d_offset"][b], [res["d_defocus"][b]]])
        for sl in (slice(0, 4), slice(4, 6), slice(6, 7)):
            err = np.linalg.norm(g_gpu[sl] - g_fd[sl]) / max(np.linalg.norm(g_fd[sl]), 1e-30)
            assert err <= GRAD_TOL, (b, sl, g_gpu[sl], g_fd[sl], err)


@pytest.mark.parametrize("box,shape,kv", [
    (32, (32, 32), 20.0),   # crop 64 -> 32, strong curvature
    (32, (40, 24), 60.0),   # non-square crop
    (32, (70, 66), 40.0),   # pad 64 -> 70 x 66
    (31, (31, 31), 30.0),   # N = 62, odd image (no Nyquist column or row)
    (64, (64, 64), 40.0),   # crop 128 -> 64: register transforms of 64 and 128 points in all three adjoint passes
])
def test_ewald_loss_and_parameter_gradients(cuda_device, box, shape, kv):
    from cryojax_b200.gradients import squared_residual_and_grad

    grid, og, fs, specs, obs = _setup(box, shape, 3, seed=box + int(kv), kv=kv)
    res = squared_residual_and_grad(_model(grid, specs), obs, grid_grad=False)
    assert res["d_rotation"].shape == (3, 3, 3)
    # the surface's curvature gives R's third column a (small: w grows as |q|^2, the signal sits at low |q|)
    # share of the gradient; the central differences below check it through the quaternion
    assert np.abs(res["d_rotation"][:, :, 2]).max() > 1e-5 * np.abs(res["d_rotation"][:, :, :2]).max()
    _check_parameter_gradients(res, og, fs, specs, obs, spline=False)


def test_ewald_spline_parameter_gradients(cuda_device):
    from cryojax_b200.gradients import squared_residual_and_grad

    grid, og, fs, specs, obs = _setup(32, (32, 32), 2, seed=41, kv=20.0, spline=True)
    res = squared_residual_and_grad(_model(grid, specs, layout="bricked", spline=True), obs, grid_grad=False)
    _check_parameter_gradients(res, og, fs, specs, obs, spline=True)


def test_ewald_grid_gradient_scatter(cuda_device):
    """Grid-gradient entries one by one (the loss is exactly quadratic in each grid value): the 10 largest and
    20 random entries above 1 % of the largest, against central differences of the oracle."""
    from cryojax_b200.gradients import squared_residual_and_grad

    grid, og, fs, specs, obs = _setup(32, (32, 32), 2, seed=9, kv=20.0)
    res = squared_residual_and_grad(_model(grid, specs), obs, grid_grad=True)
    gg = res["d_grid"].cpu().numpy()
    mag = np.abs(gg).ravel()
    scale = mag.max()
    rng = np.random.default_rng(0)
    big = np.flatnonzero(mag >= 0.01 * scale)
    idxs = list(np.argsort(mag)[::-1][:10]) + list(rng.choice(big, 20, replace=False))
    for flat_i in idxs:
        z, y, x = np.unravel_index(flat_i, gg.shape)
        h = 1e-2 * max(abs(grid[z, y, x]), 1.0)

        def loss_at(d):
            g2 = grid.copy()
            g2[z, y, x] += d
            return _loss(g2, fs, specs, obs)

        fd = (loss_at(h) - loss_at(-h)) / (2 * h) + 1j * (loss_at(1j * h) - loss_at(-1j * h)) / (2 * h)
        assert abs(gg[z, y, x] - fd) <= GRAD_TOL * abs(fd), ((z, y, x), gg[z, y, x], fd)
        assert abs(gg[z, y, x] - fd) <= GRAD_TOL * scale


@pytest.mark.parametrize("layout", ["linear", "bricked"])
def test_ewald_grid_layouts_give_same_gradients(cuda_device, layout):
    from cryojax_b200.gradients import squared_residual_and_grad

    grid, _, _, specs, obs = _setup(32, (32, 32), 2, seed=12, kv=30.0)
    ref = squared_residual_and_grad(_model(grid, specs, layout="pairs"), obs, grid_grad=True)
    got = squared_residual_and_grad(_model(grid, specs, layout=layout), obs, grid_grad=True)
    np.testing.assert_allclose(got["loss"], ref["loss"], rtol=1e-6)
    np.testing.assert_allclose(got["d_wxyz"], ref["d_wxyz"], rtol=1e-4, atol=1e-6 * np.abs(ref["d_wxyz"]).max())
    a, b = got["d_grid"].cpu().numpy(), ref["d_grid"].cpu().numpy()
    assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max()
