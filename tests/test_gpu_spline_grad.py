"""GPU: loss gradients through a FourierVoxelSplineVolume against float64 central differences of the oracle.

Same construction as the trilinear gradient tests: observed images are the
oracle's spline simulations at a true pose plus white noise, the loss is
taken at a perturbed pose.  The cubic spline is C2, so central
differences need no care at cell boundaries (step 1e-6 on the quaternion,
1e-4 on offsets, defocus and coefficients).  Tolerances: loss rel 1e-5;
each gradient group rel L2 1e-4; coefficient-gradient entries within 1e-4
of the largest.
"""

import copy

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import make_volume, specs_to_model_args

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4


def _loss(coef, fs, specs, obs):
    return sum(float(np.sum((O.simulate(coef, fs, s, spline=True) - o) ** 2)) for s, o in zip(specs, obs))


def _fd(f, h):
    return (f(h) - f(-h)) / (2 * h)


def _setup(seed, n=2, box=32):  # N = 64, images 32^2: the loss gradient's register-FFT sizes (32 R)
    rng = np.random.default_rng(seed)
    _, grid, fs = make_volume(box, 50, seed=seed)
    coef = O.compute_spline_coefficients(grid)
    true_q, off = O.uniform_poses(n, seed + 1, 8.0)
    specs, obs = [], []
    for b in range(n):
        s_true = O.ImageSpec(shape=(box, box), pixel_size=2.0, wxyz=true_q[b], offset_in_angstroms=off[b],
                             defocus_in_angstroms=rng.uniform(8000, 15000), astigmatism_in_angstroms=150.0,
                             astigmatism_angle=30.0)
        img = O.simulate(coef, fs, s_true, spline=True)
        obs.append(img + rng.standard_normal(img.shape) * np.sqrt(img.var() / 0.1))
        axis = rng.standard_normal(3)
        axis /= np.linalg.norm(axis)
        s = copy.deepcopy(s_true)
        s.wxyz = O.quat_compose(O.so3_exp(np.deg2rad(rng.uniform(0.5, 3.0)) * axis), true_q[b])
        s.offset_in_angstroms = off[b] + rng.uniform(-2, 2, 2)
        s.defocus_in_angstroms = s_true.defocus_in_angstroms + rng.uniform(-300, 300)
        specs.append(s)
    return coef, fs, specs, np.stack(obs)


def _model(coef, specs, bricked=True):
    import torch

    from cryojax_b200 import simulator as S

    pose, tt, cfg = specs_to_model_args(specs)
    vol = S.FourierVoxelSplineVolume(torch.as_tensor(coef.astype(np.complex64)).cuda())
    model = S.make_image_model(vol, cfg, pose, tt)
    model.volume_integrator.use_bricked_layout = bricked
    return model


def test_spline_loss_and_pose_gradients(cuda_device):
    from cryojax_b200.gradients import squared_residual_and_grad

    coef, fs, specs, obs = _setup(seed=3)
    res = squared_residual_and_grad(_model(coef, specs), obs, grid_grad=False)
    for b, s in enumerate(specs):
        ref = _loss(coef, fs, [s], obs[b:b + 1])
        assert abs(res["loss"][b] - ref) <= 1e-5 * ref

        def with_(fn, h):
            s2 = copy.deepcopy(s)
            fn(s2, h)
            return _loss(coef, fs, [s2], obs[b:b + 1])

        g = [_fd(lambda h, c=c: with_(lambda s2, h: setattr(s2, "wxyz", s.wxyz + h * np.eye(4)[c]), h), 1e-6)
             for c in range(4)]
        g += [_fd(lambda h: with_(lambda s2, h: setattr(s2, "offset_in_angstroms", s.offset_in_angstroms + [h, 0]),
                                  h), 1e-4),
              _fd(lambda h: with_(lambda s2, h: setattr(s2, "offset_in_angstroms", s.offset_in_angstroms + [0, h]),
                                  h), 1e-4),
              _fd(lambda h: with_(lambda s2, h: setattr(s2, "defocus_in_angstroms", s.defocus_in_angstroms + h), h),
                  1e-4)]
        g = np.array(g)
        got = np.concatenate([res["d_wxyz"][b], res["d_offset"][b], [res["d_defocus"][b]]])
        for sl in (slice(0, 4), slice(4, 6), slice(6, 7)):
            err = np.linalg.norm(got[sl] - g[sl]) / max(np.linalg.norm(g[sl]), 1e-30)
            assert err <= GRAD_TOL, (b, sl, got[sl], g[sl], err)


def test_spline_coefficient_gradient_and_layouts(cuda_device):
    from cryojax_b200.gradients import squared_residual_and_grad

    coef, fs, specs, obs = _setup(seed=7)
    out = [squared_residual_and_grad(_model(coef, specs, bricked), obs, grid_grad=True) for bricked in (True, False)]
    gg = out[0]["d_grid"].cpu().numpy()
    assert gg.shape == coef.shape
    assert np.abs(gg - out[1]["d_grid"].cpu().numpy()).max() <= 1e-5 * np.abs(gg).max()
    np.testing.assert_allclose(out[0]["d_wxyz"], out[1]["d_wxyz"], rtol=1e-5, atol=1e-8 * np.abs(out[1]["d_wxyz"]).max())
    scale = np.abs(gg).max()
    rng = np.random.default_rng(1)
    idxs = list(np.argsort(np.abs(gg).ravel())[::-1][:4]) + list(rng.choice(np.flatnonzero(np.abs(gg) > 0), 3))
    for flat_i in idxs:
        z, y, x = np.unravel_index(flat_i, gg.shape)

        def loss_at(h, part):
            c2 = coef.copy()
            c2[z, y, x] += h * (1.0 if part == 0 else 1.0j)
            return _loss(c2, fs, specs, obs)

        fd = _fd(lambda h: loss_at(h, 0), 1e-4) + 1j * _fd(lambda h: loss_at(h, 1), 1e-4)
        assert abs(gg[z, y, x] - fd) <= GRAD_TOL * scale, ((z, y, x), gg[z, y, x], fd, scale)
