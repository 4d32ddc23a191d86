"""GPU: noise model statistics and log-likelihood against the oracle's formulas."""

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import make_volume, random_specs, specs_to_model_args

pytestmark = pytest.mark.gpu


def test_noise_statistics_and_log_likelihood(cuda_device):
    import torch

    from cryojax_b200 import simulator as S
    from cryojax_b200.noise import GaussianWhiteNoiseModel

    vol, grid, fs = make_volume(32, 40, seed=4)
    specs = random_specs(64, seed=5, shape=(32, 32))
    pose, tt, cfg = specs_to_model_args(specs)
    model = S.make_image_model(S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda()),
                               cfg, pose, tt)
    nm = GaussianWhiteNoiseModel(model, variance=2.5)
    g = torch.Generator(device="cuda").manual_seed(0)
    noise = nm.compute_noise(g).cpu().numpy()
    # real-space per-pixel variance of the reference's recipe: var * (1 - 1/P^2) on average
    assert abs(noise.var() / 2.5 - 1.0) < 0.05
    assert abs(noise.mean()) < 0.02
    obs = nm.sample(g).cpu().numpy()
    ll = nm.log_likelihood(torch.as_tensor(obs).cuda()).cpu().numpy()
    sim = np.stack([O.simulate(grid, fs, s) for s in specs])
    ref = [O.gaussian_white_log_likelihood(sim[b], obs[b], 2.5) for b in range(len(specs))]
    np.testing.assert_allclose(ll, ref, rtol=1e-6)
