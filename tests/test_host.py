"""Host-side logic of the simulator mirror (no GPU): parameter packing, rotations, ordering."""

import numpy as np
import pytest

from cryojax_b200 import _native as nat
from cryojax_b200 import rotations as rot
from cryojax_b200 import simulator as S
from oracle import cryojax_oracle as O


def test_rotations_match_oracle():
    rng = np.random.default_rng(0)
    q = rng.standard_normal((5, 4))
    for b in range(5):
        np.testing.assert_allclose(rot.quat_to_matrix(q[b]), O.quat_as_matrix(q[b]), atol=1e-14)
    e = rng.uniform(-180, 180, (5, 3))
    qe = rot.euler_zyz_to_quat(e[:, 0], e[:, 1], e[:, 2])
    for b in range(5):
        np.testing.assert_allclose(qe[b], O.euler_pose_quaternion(*e[b]), atol=1e-14)
    ev = rng.uniform(-90, 90, (5, 3))
    for b in range(5):
        np.testing.assert_allclose(rot.so3_exp(np.deg2rad(ev[b])), O.axis_angle_pose_quaternion(ev[b]), atol=1e-14)


def test_pose_parametrisations_agree_on_rotation():
    wxyz = np.array([1.0, 2.0, 3.0, 0.5])
    p = S.QuaternionPose(wxyz=wxyz)
    r = p.rotation_matrices()
    theta = np.arccos(r[2, 2])
    phi = np.arctan2(r[2, 1], -r[2, 0])
    psi = np.arctan2(r[1, 2], r[0, 2])
    e = S.EulerAnglePose(phi_angle=np.rad2deg(phi), theta_angle=np.rad2deg(theta), psi_angle=np.rad2deg(psi))
    np.testing.assert_allclose(e.rotation_matrices(), r, atol=1e-12)


def test_pack_image_params_fields():
    pose = S.EulerAnglePose(1.5, -2.0, 10.0, 20.0, 30.0, offset_z_in_angstroms=50.0)
    ctf = S.AstigmaticCTF(9800.0, 200.0, 10.0, 2.7)
    tt = S.ContrastTransferTheory(ctf, amplitude_contrast_ratio=0.1, phase_shift=5.0)
    cfg = S.BasicImageConfig((32, 32), 2.0, 300.0)
    p = S.pack_image_params(pose, cfg, tt, scale=3.0)
    assert p.shape == (1, nat.PARAMS_DOUBLES)
    np.testing.assert_allclose(p[0, 0:9].reshape(3, 3), O.quat_as_matrix(O.euler_pose_quaternion(10, 20, 30)),
                               atol=1e-14)
    assert p[0, nat.P_SHIFT_X] == 1.5 and p[0, nat.P_SHIFT_Y] == -2.0
    assert p[0, nat.P_DEFOCUS] == pytest.approx(9850.0)  # defocus + offset_z
    assert p[0, nat.P_CS] == pytest.approx(2.7e7)
    assert p[0, nat.P_ASTIG_ANGLE] == pytest.approx(np.deg2rad(10.0))
    assert p[0, nat.P_WAVELENGTH] == pytest.approx(float(O.wavelength_from_kilovolts(300.0)))
    assert p[0, nat.P_PHASE_TOTAL] == pytest.approx(np.deg2rad(5.0) + O.amplitude_contrast_phase_shift(0.1))
    assert p[0, nat.P_SCALE] == 3.0


def test_batched_packing_broadcasts():
    q = O.uniform_poses(7, 3, 5.0)[0]
    pose = S.QuaternionPose(np.arange(7.0), 0.0, wxyz=q)
    tt = S.ContrastTransferTheory(S.AstigmaticCTF(np.linspace(5000, 9000, 7)))
    cfg = S.BasicImageConfig((16, 16), 1.5, 200.0)
    p = S.pack_image_params(pose, cfg, tt)
    assert p.shape == (7, 32)
    np.testing.assert_allclose(p[:, nat.P_SHIFT_X], np.arange(7.0))
    np.testing.assert_allclose(p[:, nat.P_DEFOCUS], np.linspace(5000, 9000, 7))
    assert np.all(p[:, nat.P_PIXEL_SIZE] == 1.5)


def test_contrast_model_scale_and_routing():
    vol = S.FourierVoxelGridVolume(np.zeros((8, 8, 8), np.complex64))
    cfg = S.BasicImageConfig((8, 8), 2.0, 300.0)
    tt = S.ContrastTransferTheory(S.AstigmaticCTF())
    m = S.make_image_model(vol, cfg, S.EulerAnglePose(), tt, simulates_quantity=True)
    assert isinstance(m, S.ContrastImageModel)
    assert m.volume_integrator.outputs_integral is True
    np.testing.assert_allclose(m._scale(), 2.0 * O.interaction_constant_from_kilovolts(300.0))
    m2 = S.make_image_model(vol, cfg, S.EulerAnglePose(), tt)
    assert isinstance(m2, S.LinearImageModel) and m2.volume_integrator.outputs_integral is False
    assert m2._flags() == nat.CJX_APPLY_CTF | nat.CJX_APPLY_TRANSLATION
    m3 = S.make_image_model(vol, cfg, S.EulerAnglePose())
    assert isinstance(m3, S.ProjectionImageModel) and m3._flags() == nat.CJX_APPLY_TRANSLATION


def test_reference_error_behaviour():
    with pytest.raises(ValueError):
        S.FourierVoxelGridVolume.from_real_voxel_grid(np.zeros((4, 4, 4)), pad_scale=0.5, device="cpu")
    with pytest.raises(AttributeError):
        S.FourierVoxelGridVolume(np.zeros((4, 4, 5), np.complex64))
    with pytest.raises(AttributeError):
        S.BasicImageConfig((10, 10), 1.0, 300.0, pad_options=dict(shape=(8, 8)))
    with pytest.raises(ValueError):
        S.BasicImageConfig((10, 10), -1.0, 300.0)
    vol = S.FourierVoxelGridVolume(np.zeros((8, 8, 8), np.complex64))
    cfg = S.BasicImageConfig((8, 8), 2.0, 300.0)
    m = S.make_image_model(vol, cfg, S.EulerAnglePose(), translate_mode="atom")
    with pytest.raises(ValueError):
        m._flags()


def test_orientation_order_is_a_locality_preserving_permutation():
    q = O.uniform_poses(4096, 9, 0.0)[0]
    R = np.stack([O.quat_as_matrix(x) for x in q])
    order = S.orientation_order(R)
    assert sorted(order.tolist()) == list(range(4096))
    n = R[:, :, 2]
    n = np.where(n[:, 2:3] < 0, -n, n)

    def mean_step(idx):
        a, b = n[idx[:-1]], n[idx[1:]]
        return np.mean(np.arccos(np.clip(np.abs(np.sum(a * b, 1)), 0, 1)))

    assert mean_step(order) < 0.2 * mean_step(np.arange(4096))


def test_matrix_to_quat_round_trip():
    from cryojax_b200 import rotations as rot

    rng = np.random.default_rng(0)
    q = rot.sample_uniform_quaternions(rng, 500)
    q = np.concatenate([q, [[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1], [0.5, 0.5, -0.5, 0.5]]])
    q2 = rot.matrix_to_quat(rot.quat_to_matrix(q))
    q = q * np.where(q[:, :1] < 0, -1.0, 1.0)
    np.testing.assert_allclose(np.abs(np.sum(q * q2, 1)), 1.0, atol=1e-12)
    np.testing.assert_allclose(rot.quat_to_matrix(q2), rot.quat_to_matrix(q), atol=1e-12)


def test_area_downsample_reference_weights():
    """The host restatement of cjx_area_downsample's weights sums each footprint exactly."""
    H, h = 320, 128
    f = H / h
    w = np.zeros((h, H))
    for i in range(h):
        y0, y1 = i * f, (i + 1) * f
        for y in range(int(np.floor(y0)), min(H, int(np.ceil(y1)))):
            w[i, y] = max(0.0, min(y1, y + 1) - max(y0, y))
    np.testing.assert_allclose(w.sum(1), f)
    np.testing.assert_allclose(w.sum(0), 1.0)


def test_gaussian_mixture_volume_shapes_and_pose():
    import numpy as np

    from cryojax_b200 import simulator as S

    v = S.GaussianMixtureVolume(np.zeros((4, 3)), 2.0, [1.0, 2.0, 3.0, 4.0])
    assert v.amplitudes.shape == (4, 1) and v.variances[:, 0].tolist() == [1.0, 2.0, 3.0, 4.0]
    with pytest.raises(ValueError):
        S.GaussianMixtureVolume(np.zeros((2, 3)), 1.0, -1.0)
    params = {"a": np.ones((3, 5)), "b": np.full((3, 5), 8 * np.pi**2)}
    t = S.GaussianMixtureVolume.from_tabulated_parameters(np.zeros((3, 3)), params, extra_b_factors=np.zeros(3))
    np.testing.assert_allclose(t.variances, 1.0)
    pose = S.EulerAnglePose(1.0, -2.0, 30.0, 40.0, 50.0)
    p = np.random.default_rng(0).standard_normal((5, 3))
    r = S.GaussianMixtureVolume(p).rotate_to_pose(pose)
    np.testing.assert_allclose(r.positions, p @ pose.rotation_matrices().T)
    back = r.rotate_to_pose(pose, inverse=True)
    np.testing.assert_allclose(back.positions, p, atol=1e-12)
    np.testing.assert_allclose(S.GaussianMixtureVolume(p).translate_to_pose(pose).positions, p + [1.0, -2.0, 0.0])


def test_host_streaming_sub_batch_plan():
    """HostStreamingSimulator.sub_batches: sub_batch / 8, / 4, / 2, then full sub-batches, covering every
    image once in order (the plan needs no device, so the simulator is not constructed)."""
    from cryojax_b200.pipeline import HostStreamingSimulator

    sim = object.__new__(HostStreamingSimulator)
    sim.sub_batch = 2048
    plan = sim.sub_batches(16384)
    counts = [c for _, c in plan]
    assert counts[:4] == [256, 512, 1024, 2048] and max(counts) == 2048 and sum(counts) == 16384
    assert [s for s, _ in plan] == list(np.cumsum([0] + counts[:-1]))
    assert sim.sub_batches(0) == [] and sim.sub_batches(100) == [(0, 100)]
    sim.sub_batch = 3
    assert sim.sub_batches(10) == [(0, 1), (1, 2), (3, 3), (6, 3), (9, 1)]


@pytest.mark.parametrize("ewald", [False, True])
def test_rotation_step_gradient_is_the_derivative_along_the_step(ewald):
    """refine's rotation step R -> exp([w]x) R: for a loss linear in R with dL/dR = G (the columns the gradient
    record holds: 0 and 1, and 2 on the Ewald sphere), dL/dw at w = 0 equals central differences of
    L(exp([w]x) R)."""
    from cryojax_b200.refine import _exp_so3, rotation_step_gradient

    rng = np.random.default_rng(3)
    n = 4
    R = rot.quat_to_matrix(rot.quat_normalize(rng.standard_normal((n, 4))))
    G = rng.standard_normal((n, 3, 3))
    if not ewald:
        G[:, :, 2] = 0.0
    g = np.zeros((n, nat.GRAD_DOUBLES))
    g[:, nat.G_ROT:nat.G_ROT + 6] = G[:, :, 0:2].reshape(n, 6)
    g[:, nat.G_ROT + 6:nat.G_ROT + 9] = G[:, :, 2]
    gw = rotation_step_gradient(R, g, ewald)
    h = 1e-6
    for a in range(3):
        w = np.zeros((n, 3))
        w[:, a] = h
        lp = np.einsum("nij,nij->n", G, _exp_so3(w) @ R)
        lm = np.einsum("nij,nij->n", G, _exp_so3(-w) @ R)
        np.testing.assert_allclose(gw[:, a], (lp - lm) / (2 * h), rtol=1e-6, atol=1e-8)
