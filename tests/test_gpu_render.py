"""GPU parity: GaussianMixtureRenderFn (cjx_render_gaussians) against the oracle's dense float64 restatement.

Tolerance: relative L2 over the grid <= 1e-5 (float32 erf integrals and
float atomics; the oracle evaluates every voxel against every Gaussian).
Cases: 1 and 5 Gaussians per atom, atoms near and beyond the faces, a
window wider than the 64-voxel shared-memory sub-box, accumulation, no
atoms, and the Fourier outputs of the render function.
"""

import numpy as np
import pytest

from oracle import cryojax_oracle as O

pytestmark = pytest.mark.gpu


def _atoms(n, g, seed, spread, var_range):
    rng = np.random.default_rng(seed)
    return (rng.uniform(-spread, spread, (n, 3)), rng.uniform(0.2, 2.0, (n, g)), rng.uniform(*var_range, (n, g)))


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("shape,dx,n,g,spread,var", [
    ((24, 28, 20), 0.9, 40, 5, 12.0, (0.2, 1.5)),    # 5 Gaussians, atoms straddling the faces
    ((32, 32, 32), 1.0, 25, 1, 10.0, (0.5, 2.0)),    # one Gaussian per atom
    ((80, 72, 76), 0.25, 3, 2, 3.0, (6.0, 9.0)),     # windows wider than a 64-voxel sub-box
    ((16, 16, 16), 1.0, 10, 3, 40.0, (0.3, 0.8)),    # most atoms far outside the grid
])
def test_render_matches_oracle(cuda_device, shape, dx, n, g, spread, var):
    from cryojax_b200 import simulator as S

    pos, amp, v = _atoms(n, g, seed=n + g, spread=spread, var_range=var)
    got = S.GaussianMixtureRenderFn(shape, dx)(S.GaussianMixtureVolume(pos, amp, v)).cpu().numpy()
    ref = O.render_gaussian_mixture(shape, dx, pos, amp, v)
    assert got.shape == ref.shape
    if np.abs(ref).max() == 0:
        assert np.abs(got).max() == 0
    else:
        assert _rel(got, ref) <= 1e-5, _rel(got, ref)


def test_accumulate_empty_and_fourier_outputs(cuda_device):
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200 import simulator as S

    pos, amp, v = _atoms(20, 5, seed=3, spread=8.0, var_range=(0.3, 1.2))
    shape, dx = (24, 24, 24), 1.0
    fn = S.GaussianMixtureRenderFn(shape, dx)
    ref = O.render_gaussian_mixture(shape, dx, pos, amp, v)
    t = lambda a: torch.as_tensor(a, dtype=torch.float32, device="cuda")
    half = nat.render_gaussians(shape, dx, t(pos[:10]), t(amp[:10]), t(v[:10]))
    nat.render_gaussians(shape, dx, t(pos[10:]), t(amp[10:]), t(v[10:]), out=half, accumulate=True)
    assert _rel(half.cpu().numpy(), ref) <= 1e-5
    empty = nat.render_gaussians(shape, dx, t(np.zeros((0, 3))), t(np.zeros((0, 5))), t(np.ones((0, 5))))
    assert torch.count_nonzero(empty) == 0
    vol = S.GaussianMixtureVolume(pos, amp, v)
    ft = fn(vol, outputs_real_space=False, fftshifted=True).cpu().numpy()
    np.testing.assert_allclose(ft, np.fft.fftshift(O.fftn(ref)), atol=1e-5 * np.abs(ft).max())
    rft = fn(vol, outputs_real_space=False, outputs_rfft=True).cpu().numpy()
    np.testing.assert_allclose(rft, O.rfftn(ref), atol=1e-5 * np.abs(rft).max())


def test_rendered_volume_feeds_the_slice_path(cuda_device):
    """A rendered volume through FourierVoxelGridVolume.from_real_voxel_grid and the forward kernels, against
    the oracle simulating the oracle's rendering."""
    from cryojax_b200 import simulator as S
    from tests.helpers import IMAGE_REL_L2_TOL, random_specs, rel_l2_per_image, specs_to_model_args

    pos, amp, v = _atoms(60, 5, seed=8, spread=10.0, var_range=(0.5, 2.0))
    shape, dx = (32, 32, 32), 2.0
    real = S.GaussianMixtureRenderFn(shape, dx)(S.GaussianMixtureVolume(pos, amp, v))
    vol = S.FourierVoxelGridVolume.from_real_voxel_grid(real, pad_scale=2.0)
    ref_real = O.render_gaussian_mixture(shape, dx, pos, amp, v)
    grid, fs = O.fourier_voxel_grid_from_real_voxel_grid(ref_real, pad_scale=2.0)
    specs = random_specs(4, seed=9, shape=(32, 32))
    pose, tt, cfg = specs_to_model_args(specs)
    got = S.make_image_model(vol, cfg, pose, tt).compute_fourier_image().cpu().numpy()
    ref = np.stack([O.compute_fourier_image(grid, fs, s) for s in specs])
    assert max(rel_l2_per_image(got, ref)) <= 2 * IMAGE_REL_L2_TOL
