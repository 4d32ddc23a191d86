"""GPU parity: simulate with a Fourier filter (fused into the device epilogue) and a real-space mask,
normalisation, and the coloured Gaussian noise model, against the float64 oracle.

Tolerances: images rel-L2 <= 1e-5 per image; log-likelihoods rel 2e-5;
the noise power spectrum within 5 % of the variance function (a
statistical check over 512 draws).
"""

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import IMAGE_REL_L2_TOL, make_volume, random_specs, rel_l2_per_image, specs_to_model_args

pytestmark = pytest.mark.gpu


def _model(grid, specs, *, normalizes=False, integrator=None):
    import torch

    from cryojax_b200 import simulator as S

    pose, tt, cfg = specs_to_model_args(specs)
    vol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
    return S.make_image_model(vol, cfg, pose, tt, normalizes_signal=normalizes, volume_integrator=integrator)


@pytest.mark.parametrize("shape,padded,normalizes", [((32, 32), None, False), ((30, 30), (40, 36), False),
                                                     ((32, 32), None, True), ((24, 28), (32, 32), True)])
def test_filter_and_mask(cuda_device, shape, padded, normalizes):
    from cryojax_b200 import transforms as T

    _, grid, fs = make_volume(32, 60, seed=5)
    specs = random_specs(4, seed=6, shape=shape, padded_shape=padded)
    ps = specs[0].padded_shape
    filt = T.LowpassFilter(T.make_frequency_grid(ps, 2.0), 2.0, 0.6, 0.1)
    mask = T.CircularCosineMask(T.make_coordinate_grid(shape, 2.0), radius=18.0, rolloff_width=6.0)
    model = _model(grid, specs, normalizes=normalizes)
    got = model.simulate(mask=mask, filter=filt).cpu().numpy()
    ref = np.stack([O.simulate(grid, fs, s, mask=mask.get(), filter=filt.get(), normalizes_signal=normalizes)
                    for s in specs])
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL
    # the filter alone is the unfiltered Fourier image times the array
    f_only = model.compute_fourier_image(filter=filt).cpu().numpy()
    plain = model.compute_fourier_image().cpu().numpy()
    np.testing.assert_allclose(f_only, plain * filt.get().astype(np.float32), rtol=0, atol=1e-6 * np.abs(plain).max())
    with pytest.raises(ValueError):
        model.simulate(filter=T.CustomFilter(np.ones((5, 5))))


def test_filter_on_the_ewald_path(cuda_device):
    from cryojax_b200 import simulator as S
    from cryojax_b200 import transforms as T

    _, grid, fs = make_volume(32, 60, seed=7)
    specs = random_specs(3, seed=8, shape=(32, 32))
    filt = T.HighpassFilter(T.make_frequency_grid((32, 32), 2.0), 2.0, 0.05, 0.05)
    model = _model(grid, specs, integrator=S.EwaldSphereExtraction(outputs_integral=False))
    got = model.simulate(filter=filt).cpu().numpy()
    ref = np.stack([O.simulate(grid, fs, s, filter=filt.get(), ewald=True) for s in specs])
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


def test_colored_noise_log_likelihood(cuda_device):
    import torch

    from cryojax_b200 import noise
    from cryojax_b200 import simulator as S

    _, grid, fs = make_volume(32, 60, seed=9)
    specs = random_specs(3, seed=10, shape=(32, 32))
    model = _model(grid, specs)
    nm = noise.GaussianColoredNoiseModel(model, S.FourierGaussian(2.0, 40.0), signal_scale_factor=1.5,
                                         signal_offset=0.1)
    rng = np.random.default_rng(0)
    observed = rng.standard_normal((3, 32, 17)) + 1j * rng.standard_normal((3, 32, 17))
    got = nm.log_likelihood(torch.as_tensor(observed).cuda()).cpu().numpy()
    var = S.FourierGaussian(2.0, 40.0)(O.make_frequency_grid((32, 32), 2.0))
    for b, s in enumerate(specs):
        sim = O.rfftn(1.5 * O.simulate(grid, fs, s) + 0.1)
        ref = O.gaussian_colored_log_likelihood(sim, observed[b], var, 32 * 32)
        np.testing.assert_allclose(got[b], ref, rtol=2e-5)  # float32 images against float64


def test_colored_noise_power_spectrum(cuda_device):
    import torch

    from cryojax_b200 import noise
    from cryojax_b200 import simulator as S
    from cryojax_b200 import transforms as T

    _, grid, fs = make_volume(16, 20, seed=11)
    specs = random_specs(512, seed=12, shape=(32, 32))
    model = _model(grid, specs)
    env = S.FourierGaussian(3.0, 60.0)
    nm = noise.GaussianColoredNoiseModel(model, env)
    gen = torch.Generator(device="cuda").manual_seed(1)
    n = nm.compute_noise(gen, outputs_real_space=False).cpu().numpy()  # [512, 32, 17]
    power = (np.abs(n) ** 2).mean(axis=0) / (32 * 32)
    expect = env(T.make_frequency_grid((32, 32), 2.0))
    ring = np.hypot(*np.meshgrid(np.arange(17), np.fft.fftfreq(32) * 32))
    for r0 in (2, 6, 10, 14):
        sel = (ring >= r0) & (ring < r0 + 2)
        assert abs(power[sel].mean() / expect[sel].mean() - 1.0) < 0.05, r0
