"""GPU parity at the benchmark configurations' sizes (register-FFT resize path).

The Fourier grids here are synthetic (seeded complex Gaussian noise under a
Gaussian envelope, so the spectrum decays like a real molecule's): the
oracle and the kernels take the grid as their input, and building it this
way avoids a float64 N^3 FFT per test.  Tolerance: relative L2 <= 1e-5 per
image against the float64 oracle.
"""

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import IMAGE_REL_L2_TOL, random_specs, rel_l2_per_image, specs_to_model_args

pytestmark = pytest.mark.gpu


def synthetic_grid(n, seed, width=0.12):
    rng = np.random.default_rng(seed)
    k = (np.arange(n) - n // 2) / n
    env1 = np.exp(-(k**2) / (2 * width**2))
    env = env1[:, None, None] * env1[None, :, None] * env1[None, None, :]
    g = rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))
    g *= env
    g[n // 2, n // 2, n // 2] += 50.0
    return g


# (N, image shape, padded shape)
CASES = [
    (128, (64, 64), None),
    (160, (96, 96), None),
    (192, (160, 160), None),
    (256, (128, 128), None),
    (256, (300, 150), (320, 160)),  # pad y (Py > N), crop x
    (320, (192, 192), None),
    (384, (192, 192), None),
    (512, (320, 320), None),        # the benchmark shape
    (512, (256, 256), None),
]


@pytest.mark.parametrize("n,shape,padded", CASES)
def test_resize_path_sizes(cuda_device, n, shape, padded):
    import torch

    from cryojax_b200 import simulator as S

    grid = synthetic_grid(n, seed=n)
    fs = O.make_frequency_slice((n, n), outputs_rfftfreqs=False)
    specs = random_specs(2, seed=n + 1, shape=shape, padded_shape=padded)
    pose, tt, cfg = specs_to_model_args(specs)
    vol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
    model = S.make_image_model(vol, cfg, pose, tt)
    got = model.compute_fourier_image().cpu().numpy()
    ref = np.stack([O.compute_fourier_image(grid, fs, s) for s in specs])
    errs = rel_l2_per_image(got, ref)
    print(f"N={n} shape={shape} padded={padded}: max rel-L2 {max(errs):.3e}")  # shown with pytest -s
    assert max(errs) <= IMAGE_REL_L2_TOL, errs


@pytest.mark.parametrize("fft_mode", [0, 1, 2, 3])
def test_fft_modes_at_the_benchmark_shape(cuda_device, fft_mode):
    """N = 512 -> 320^2 through each FFT implementation (Stockham, shuffle network, 512-point transpose)."""
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200 import simulator as S

    n, shape = 512, (320, 320)
    grid = synthetic_grid(n, seed=77)
    fs = O.make_frequency_slice((n, n), outputs_rfftfreqs=False)
    specs = random_specs(2, seed=78, shape=shape)
    pose, tt, cfg = specs_to_model_args(specs)
    vol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
    old = nat.tuning_get(nat.CJX_TUNE_FFT_MODE)
    try:
        nat.tuning_set(nat.CJX_TUNE_FFT_MODE, fft_mode)
        got = S.make_image_model(vol, cfg, pose, tt).compute_fourier_image().cpu().numpy()
    finally:
        nat.tuning_set(nat.CJX_TUNE_FFT_MODE, old)
    ref = np.stack([O.compute_fourier_image(grid, fs, s) for s in specs])
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL
