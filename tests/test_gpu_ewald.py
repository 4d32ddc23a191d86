"""GPU parity: EwaldSphereExtraction (CJX_EWALD_SPHERE) through the C-ABI against the float64 oracle.

The integrator's full spectrum and the non-projection contrast of
ContrastTransferTheory, for crop, pad, odd and prime N, the no-resize path,
trilinear and spline volumes in every layout, the contrast model with
envelope and defocus offset.  Tolerance: relative L2 error per image
IMAGE_REL_L2_TOL (1e-5), as for the slice path.  Low accelerating voltages
(larger wavelengths) are included so that the sphere's curvature moves the
samples by up to a voxel.
"""

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import IMAGE_REL_L2_TOL, make_volume, rel_l2_per_image, specs_to_model_args

pytestmark = pytest.mark.gpu


def _specs(n, seed, shape, padded=None, kv=300.0, pixel_size=2.0, offset_z=False, envelope=False):
    rng = np.random.default_rng(seed)
    q, off = O.uniform_poses(n, seed + 1, 8.0)
    out = []
    for b in range(n):
        o = np.array([off[b][0], off[b][1], rng.uniform(-300, 300)]) if offset_z else off[b]
        out.append(O.ImageSpec(
            shape=shape, padded_shape=padded, pixel_size=pixel_size, voltage_in_kilovolts=kv, wxyz=q[b],
            offset_in_angstroms=o, defocus_in_angstroms=rng.uniform(5000, 25000),
            astigmatism_in_angstroms=rng.uniform(0, 500), astigmatism_angle=rng.uniform(0, 180),
            spherical_aberration_in_mm=2.7, amplitude_contrast_ratio=rng.uniform(0.05, 0.2),
            phase_shift=rng.uniform(0, 20), envelope_b_factor=(rng.uniform(20, 80) if envelope else None)))
    return out


def _volume(grid, spline):
    import torch

    from cryojax_b200 import simulator as S

    v = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
    return S.FourierVoxelSplineVolume.from_fourier_voxel_grid(v) if spline else v


def _integrator(layout, **kw):
    from cryojax_b200 import simulator as S

    return S.EwaldSphereExtraction(use_bricked_layout=layout != "linear", pair_layout=layout == "pairs", **kw)


def _model(vol, specs, integ, quantity=False):
    from cryojax_b200 import simulator as S

    pose, tt, cfg = specs_to_model_args(specs)
    return S.make_image_model(vol, cfg, pose, tt, volume_integrator=integ, simulates_quantity=quantity)


def _oracle_grid(grid, spline):
    return O.compute_spline_coefficients(grid) if spline else grid


CASES = [
    # (box, pad_scale, shape, padded_shape, kV)
    (32, 2.0, (32, 32), None, 300.0),      # crop 64 -> 32
    (32, 2.0, (64, 64), None, 300.0),      # no resize
    (32, 2.0, (70, 66), None, 300.0),      # pad
    (32, 2.0, (40, 24), None, 20.0),       # non-square crop, strong curvature
    (25, 1.0, (25, 25), None, 20.0),       # odd N, no resize
    (32, 1.3, (30, 30), (44, 42), 60.0),   # prime N = 41, padded != shape
    (31, 2.0, (31, 31), None, 300.0),      # N = 62, odd image
    (32, 2.0, (64, 33), None, 60.0),       # register column pass (Py = 64), odd Px
    (32, 2.0, (32, 40), None, 300.0),      # register column pass, Px = 40 (shared-memory rows)
]


@pytest.mark.parametrize("box,pad_scale,shape,padded,kv", CASES)
@pytest.mark.parametrize("layout", ["linear", "pairs"])
@pytest.mark.parametrize("spline", [False, True])
def test_ewald_image_model_matches_oracle(cuda_device, box, pad_scale, shape, padded, kv, layout, spline):
    _, grid, fs = make_volume(box, 60, seed=box + 5, pad_scale=pad_scale)
    specs = _specs(4, seed=2 * box, shape=shape, padded=padded, kv=kv)
    vol = _volume(grid, spline)
    model = _model(vol, specs, _integrator(layout, outputs_integral=False))
    got = model.compute_fourier_image().cpu().numpy()
    og = _oracle_grid(grid, spline)
    ref = np.stack([O.compute_fourier_image(og, fs, s, ewald=True, spline=spline) for s in specs])
    assert got.shape == ref.shape
    errs = rel_l2_per_image(got, ref)
    assert max(errs) <= IMAGE_REL_L2_TOL, errs
    # it is not the projection image
    proj = np.stack([O.compute_fourier_image(og, fs, s, spline=spline) for s in specs])
    assert min(rel_l2_per_image(proj, ref)) > 1e-4


@pytest.mark.parametrize("shape,padded", [((32, 32), None), ((64, 64), None), ((30, 30), (36, 34))])
@pytest.mark.parametrize("bricked", [False, True])
def test_integrate_gives_the_full_spectrum(cuda_device, shape, padded, bricked):
    from cryojax_b200 import simulator as S

    _, grid, fs = make_volume(32, 60, seed=9)
    specs = _specs(3, seed=4, shape=shape, padded=padded, kv=30.0)
    pose, _, cfg = specs_to_model_args(specs)
    vol = _volume(grid, False).rotate_to_pose(pose)
    integ = S.EwaldSphereExtraction(outputs_integral=True, use_bricked_layout=bricked, pair_layout=False)
    got = integ.integrate(vol, cfg).cpu().numpy()
    wl = O.wavelength_from_kilovolts(30.0)
    ref = np.stack([O.ewald_integrate(grid, O.rotate_frequency_slice(fs, O.quat_normalize(s.wxyz)), s.padded_shape,
                                      s.pixel_size, wl, outputs_integral=True) for s in specs])
    assert got.shape == ref.shape == (3,) + tuple(specs[0].padded_shape)
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


@pytest.mark.parametrize("shape", [(32, 32), (64, 64)])
def test_contrast_model_envelope_offset_z_and_fill(cuda_device, shape):
    _, grid, fs = make_volume(32, 60, seed=13, sigma_range=(0.5, 0.9))
    specs = _specs(4, seed=17, shape=shape, kv=40.0, offset_z=True, envelope=True)
    fill = 0.1 - 0.2j
    model = _model(_volume(grid, False), specs, _integrator("pairs", outputs_integral=True, fill_value=fill),
                   quantity=True)
    got = model.compute_fourier_image().cpu().numpy()
    ref = np.stack([O.compute_fourier_image(grid, fs, s, ewald=True, outputs_integral=True, simulates_quantity=True,
                                            cval=fill) for s in specs])
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


def test_ewald_simulate_real_space(cuda_device):
    _, grid, fs = make_volume(32, 60, seed=3)
    specs = _specs(3, seed=5, shape=(30, 30), padded=(40, 40), kv=60.0)
    model = _model(_volume(grid, False), specs, _integrator("pairs", outputs_integral=True))
    got = model.simulate().cpu().numpy()
    ref = np.stack([O.simulate(grid, fs, s, ewald=True, outputs_integral=True) for s in specs])
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


def test_ewald_rejections(cuda_device):
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200 import simulator as S

    _, grid, fs = make_volume(16, 20, seed=2)
    specs = _specs(2, seed=3, shape=(16, 16))
    pose, tt, cfg = specs_to_model_args(specs)
    vol = _volume(grid, False)
    proj = S.make_image_model(vol, cfg, pose, None, volume_integrator=S.EwaldSphereExtraction())
    with pytest.raises(NotImplementedError):
        proj.compute_fourier_image()
    with pytest.raises(nat.CryojaxB200Error) as e:
        nat.workspace_size(nat.make_desc(32, 16, 16, nat.CJX_EWALD_SPHERE | nat.CJX_APPLY_TRANSLATION), 1)
    assert e.value.code == nat.CJX_ERR_INVALID_ARGUMENT
    # the loss gradient is on the contrast image: the bare spectrum has none
    with pytest.raises(nat.CryojaxB200Error) as e:
        nat.loss_workspace_size(nat.make_desc(32, 16, 16, nat.CJX_EWALD_SPHERE), 1)
    assert e.value.code == nat.CJX_ERR_UNSUPPORTED
    assert nat.loss_workspace_size(nat.make_desc(32, 16, 16, nat.CJX_EWALD_SPHERE | nat.CJX_APPLY_CTF), 1) > 0
    torch.cuda.synchronize()


@pytest.mark.parametrize("spline", [False, True])
def test_register_fft_passes_match_oracle(cuda_device, spline):
    """N = 128 -> 96^2 (register transforms of 128 and 96 points in the row and column passes)."""
    _, grid, fs = make_volume(64, 120, seed=41)
    specs = _specs(3, seed=43, shape=(96, 96), kv=40.0)
    model = _model(_volume(grid, spline), specs, _integrator("pairs", outputs_integral=False))
    got = model.compute_fourier_image().cpu().numpy()
    og = _oracle_grid(grid, spline)
    ref = np.stack([O.compute_fourier_image(og, fs, s, ewald=True, spline=spline) for s in specs])
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


def test_fft_modes_agree_at_the_benchmark_shape(cuda_device):
    """N = 512 -> 320^2: register-FFT passes (mode 2; mode 3, the default, with the 512-point transpose FFT in
    the row pass) against the shared-memory Stockham passes (mode 0)."""
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200 import simulator as S
    from cryojax_b200 import synthetic

    vol = S.FourierVoxelGridVolume.from_real_voxel_grid(synthetic.gaussian_sum_volume(256, 2000, 3),
                                                        pad_scale=2.0)
    b = synthetic.image_batch(16, 5)
    pose = S.QuaternionPose(b.offsets[:, 0], b.offsets[:, 1], wxyz=b.wxyz)
    tt = S.ContrastTransferTheory(S.AstigmaticCTF(b.defocus, b.astigmatism, b.astigmatism_angle))
    cfg = S.BasicImageConfig((320, 320), 2.0, 300.0)
    model = S.make_image_model(vol, cfg, pose, tt, volume_integrator=S.EwaldSphereExtraction(outputs_integral=False))
    old = nat.tuning_get(nat.CJX_TUNE_FFT_MODE)
    try:
        outs = {}
        for mode in (0, 2, 3):
            nat.tuning_set(nat.CJX_TUNE_FFT_MODE, mode)
            outs[mode] = model.compute_fourier_image().cpu().numpy()
    finally:
        nat.tuning_set(nat.CJX_TUNE_FFT_MODE, old)
    torch.cuda.synchronize()
    assert max(rel_l2_per_image(outs[2], outs[0])) <= 1e-5
    assert max(rel_l2_per_image(outs[3], outs[0])) <= 1e-5  # the transpose FFT in the row pass
