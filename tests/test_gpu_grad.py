"""GPU: squared-residual loss and gradients against float64 central differences of the oracle.

Each observed image is the oracle's simulation at a seeded true pose plus
white noise.  The loss is evaluated at a perturbed pose (<= 3 deg, +-2 A,
+-300 A defocus).  Central differences use step 1e-6 on the pose (so
almost no sample crosses a voxel-cell boundary, where trilinear
interpolation has a kink) and 1e-4 on offsets, defocus and grid values.
Tolerances: loss rel 1e-5; each gradient vector (per image) rel L2 1e-4;
grid-gradient entries within 1e-4 of their own magnitude (entries above 1 %
of the largest) and of the largest.
"""

import copy

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import make_volume

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4


def _loss(grid, fs, specs, obs):
    return sum(float(np.sum((O.simulate(grid, fs, s) - o) ** 2)) for s, o in zip(specs, obs))


def _setup(box=32, shape=(32, 32), n=3, seed=0, euler=False):
    rng = np.random.default_rng(seed)
    vol, grid, fs = make_volume(box, 60, seed=seed)
    true_q, off = O.uniform_poses(n, seed + 1, 8.0)
    specs, obs = [], []
    for b in range(n):
        s_true = O.ImageSpec(shape=shape, pixel_size=2.0, wxyz=true_q[b], offset_in_angstroms=off[b],
                             defocus_in_angstroms=rng.uniform(8000, 15000), astigmatism_in_angstroms=150.0,
                             astigmatism_angle=30.0)
        img = O.simulate(grid, fs, s_true)
        noise = rng.standard_normal(img.shape) * np.sqrt(img.var() / 0.1)
        obs.append(img + noise)
        # perturbed evaluation pose: <= 3 degrees, +-2 A, +-300 A
        axis = rng.standard_normal(3)
        axis /= np.linalg.norm(axis)
        dq = O.so3_exp(np.deg2rad(rng.uniform(0.5, 3.0)) * axis)
        s = copy.deepcopy(s_true)
        s.wxyz = O.quat_compose(dq, true_q[b])
        s.offset_in_angstroms = off[b] + rng.uniform(-2, 2, 2)
        s.defocus_in_angstroms = s_true.defocus_in_angstroms + rng.uniform(-300, 300)
        specs.append(s)
    return grid, fs, specs, np.stack(obs)


def _model(grid, specs, euler=False):
    import torch

    from cryojax_b200 import simulator as S
    from tests.helpers import specs_to_model_args

    pose, tt, cfg = specs_to_model_args(specs)
    if euler:
        angles = []
        for s in specs:  # zyz Euler angles of each quaternion (extrinsic, degrees)
            r = O.quat_as_matrix(O.quat_normalize(s.wxyz))
            theta = np.arccos(np.clip(r[2, 2], -1, 1))
            phi = np.arctan2(r[2, 1], -r[2, 0])
            psi = np.arctan2(r[1, 2], r[0, 2])
            angles.append(np.rad2deg([phi, theta, psi]))
        a = np.array(angles)
        off = np.stack([s.offset_in_angstroms for s in specs])
        pose = S.EulerAnglePose(off[:, 0], off[:, 1], a[:, 0], a[:, 1], a[:, 2])
    vol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
    return S.make_image_model(vol, cfg, pose, tt), pose


def _fd(f, h):
    return (f(h) - f(-h)) / (2 * h)


@pytest.mark.parametrize("box,shape", [(32, (32, 32)), (48, (64, 64))])
def test_loss_and_parameter_gradients(cuda_device, box, shape):
    from cryojax_b200.gradients import squared_residual_and_grad

    grid, fs, specs, obs = _setup(box=box, shape=shape, seed=box)
    model, _ = _model(grid, specs)
    res = squared_residual_and_grad(model, obs, grid_grad=False)
    for b, s in enumerate(specs):
        ref_loss = _loss(grid, fs, [s], obs[b:b + 1])
        assert abs(res["loss"][b] - ref_loss) <= 1e-5 * ref_loss

        def with_(fn, h):
            s2 = copy.deepcopy(s)
            fn(s2, h)
            return _loss(grid, fs, [s2], obs[b:b + 1])

        g_fd = []
        for c in range(4):
            def fq(s2, h, c=c):
                s2.wxyz = s.wxyz + h * np.eye(4)[c]
            g_fd.append(_fd(lambda h: with_(fq, h), 1e-6))
        g_fd += [_fd(lambda h: with_(lambda s2, h: setattr(s2, "offset_in_angstroms",
                                                           s.offset_in_angstroms + [h, 0]), h), 1e-4),
                 _fd(lambda h: with_(lambda s2, h: setattr(s2, "offset_in_angstroms",
                                                           s.offset_in_angstroms + [0, h]), h), 1e-4),
                 _fd(lambda h: with_(lambda s2, h: setattr(s2, "defocus_in_angstroms",
                                                           s.defocus_in_angstroms + h), h), 1e-4)]
        g_fd = np.array(g_fd)
        g_gpu = np.concatenate([res["d_wxyz"][b], res["d_offset"][b], [res["d_defocus"][b]]])
        # per-group relative error (quaternion, offsets, defocus have different scales)
        for sl in (slice(0, 4), slice(4, 6), slice(6, 7)):
            err = np.linalg.norm(g_gpu[sl] - g_fd[sl]) / max(np.linalg.norm(g_fd[sl]), 1e-30)
            assert err <= GRAD_TOL, (b, sl, g_gpu[sl], g_fd[sl], err)


def test_euler_pose_chain(cuda_device):
    from cryojax_b200.gradients import squared_residual_and_grad

    grid, fs, specs, obs = _setup(seed=5, n=2)
    model, pose = _model(grid, specs, euler=True)
    res = squared_residual_and_grad(model, obs, grid_grad=False)
    for b, s in enumerate(specs):
        ang = np.array([pose.phi_angle[b], pose.theta_angle[b], pose.psi_angle[b]])

        def loss_at(a):
            s2 = copy.deepcopy(s)
            s2.wxyz = O.euler_pose_quaternion(*a)
            return _loss(grid, fs, [s2], obs[b:b + 1])

        g_fd = np.array([_fd(lambda h, c=c: loss_at(ang + h * np.eye(3)[c]), 1e-5) for c in range(3)])
        err = np.linalg.norm(res["d_euler_angles"][b] - g_fd) / np.linalg.norm(g_fd)
        assert err <= GRAD_TOL, (res["d_euler_angles"][b], g_fd)


def test_grid_gradient_scatter(cuda_device):
    """Grid-gradient entries one by one.  The loss is exactly quadratic in each grid value (the image is
    linear in the grid), so a central difference is exact up to rounding at any step; every checked entry
    (the 10 largest and 20 random ones among entries above 1 % of the largest) must agree to a relative
    error of 1e-4 of its own magnitude, and every entry to 1e-4 of the largest."""
    from cryojax_b200.gradients import squared_residual_and_grad

    grid, fs, specs, obs = _setup(seed=9, n=2)
    model, _ = _model(grid, specs)
    res = squared_residual_and_grad(model, obs, grid_grad=True)
    gg = res["d_grid"].cpu().numpy()
    n = grid.shape[0]
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
    assert gg.shape == (n, n, n)


@pytest.mark.parametrize("layout", ["bricked", "linear"])
def test_grid_layouts_give_same_gradients(cuda_device, layout):
    """The x-pair layout (the default), the bricked layout and the C-order array give the same loss and
    gradients up to the order of the float additions."""
    from cryojax_b200.gradients import squared_residual_and_grad

    grid, fs, specs, obs = _setup(seed=13, n=2)
    out = []
    for lay in ("pairs", layout):
        model, _ = _model(grid, specs)
        model.volume_integrator.use_bricked_layout = lay != "linear"
        model.volume_integrator.pair_layout = lay == "pairs"
        out.append(squared_residual_and_grad(model, obs, grid_grad=True))
    for key in ("loss", "d_wxyz", "d_offset", "d_defocus"):
        np.testing.assert_allclose(out[0][key], out[1][key], rtol=1e-5, atol=1e-8 * np.abs(out[1][key]).max())
    a, b = out[0]["d_grid"].cpu().numpy(), out[1]["d_grid"].cpu().numpy()
    assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max()


@pytest.mark.parametrize("mode", [1, 2])
def test_vector_atomic_scatter_matches_per_corner_atomics(cuda_device, mode):
    """16-byte x-pair atomics (mode 1) and warp-aggregated atomics (mode 2) in the grid scatter give the
    per-corner 8-byte atomics' gradient (mode 0) up to the order of the float additions."""
    from cryojax_b200 import _native as nat
    from cryojax_b200.gradients import squared_residual_and_grad

    grid, fs, specs, obs = _setup(box=48, shape=(64, 64), seed=17, n=3)
    out = []
    old = nat.tuning_get(nat.CJX_TUNE_SCATTER_VEC)
    try:
        for agg in (mode, 0):
            nat.tuning_set(nat.CJX_TUNE_SCATTER_VEC, agg)
            model, _ = _model(grid, specs)
            out.append(squared_residual_and_grad(model, obs, grid_grad=True))
    finally:
        nat.tuning_set(nat.CJX_TUNE_SCATTER_VEC, old)
    a, b = out[0]["d_grid"].cpu().numpy(), out[1]["d_grid"].cpu().numpy()
    assert np.abs(a - b).max() <= 1e-5 * np.abs(b).max()
    np.testing.assert_array_equal(out[0]["loss"], out[1]["loss"])


def _raw_loss_grad(grid, specs, obs, grid_grad, pairs):
    """One cjx_slice_ctf_loss_grad call with a caller-given grid_grad tensor."""
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200.gradients import observed_to_fourier

    model, _ = _model(grid, specs)
    integ = model.volume_integrator
    integ.pair_layout = pairs
    vol = model.volume_parametrization.get_representation()
    g, layout = integ.device_grid(vol)
    n_img = len(specs)
    py, px = model.image_config.padded_shape
    desc = nat.make_desc(vol.shape[0], py, px, model._flags() | layout)
    ws = torch.empty(nat.loss_workspace_size(desc, n_img), dtype=torch.uint8, device="cuda")
    grads = torch.empty((n_img, nat.GRAD_DOUBLES), dtype=torch.float64, device="cuda")
    pd = torch.as_tensor(model.image_params(), device="cuda")
    nat.slice_ctf_loss_grad(desc, g, pd, observed_to_fourier(obs), grads, grid_grad, ws)
    torch.cuda.synchronize()
    return grads.cpu().numpy()


@pytest.mark.parametrize("pairs", [False, True])
def test_gradient_array_only_8_byte_aligned(cuda_device, pairs):
    """A grid_grad that is only 8-byte aligned (a view one entry into a larger array) takes the 8-byte
    atomics and gives the 16-byte-aligned result; the entry before the view stays untouched."""
    import torch

    from cryojax_b200 import _native as nat

    grid, fs, specs, obs = _setup(box=48, shape=(64, 64), seed=19, n=2)
    n = grid.shape[0]
    ref = torch.zeros((n, n, n), dtype=torch.complex64, device="cuda")
    g_ref = _raw_loss_grad(grid, specs, obs, ref, pairs)
    big = torch.zeros(n ** 3 + 1, dtype=torch.complex64, device="cuda")
    shifted = big[1:].view(n, n, n)
    assert shifted.data_ptr() % 16 == 8
    g_shift = _raw_loss_grad(grid, specs, obs, shifted, pairs)
    scale = ref.abs().max().item()
    assert scale > 0
    assert (shifted - ref).abs().max().item() <= 1e-5 * scale
    np.testing.assert_array_equal(g_shift[:, nat.G_LOSS], g_ref[:, nat.G_LOSS])
    assert big[0].item() == 0
