"""GPU: cjx_postprocess_real and cjx_rfft2 (the real-space output path) against the float64 oracle.

irfftn -> centre crop -> normalise -> mask (cryojax/simulator/_image_model/base_image_model.py:107-158)
and rfftn (ifftshift, then rfft2) on random inputs over even, odd and prime sizes, crops of every parity
combination, with and without normalisation and mask; rfftn(irfftn(F)) returns F for a half plane
that is Hermitian where an inverse real FFT needs it.  Tolerance: relative L2 <= 1e-5 per image.
"""

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import IMAGE_REL_L2_TOL, rel_l2_per_image

pytestmark = pytest.mark.gpu

SHAPES = [(32, 32), (64, 40), (33, 47), (31, 31), (96, 63), (320, 320), (41, 37), (128, 256), (512, 384), (192, 96)]


def _half_planes(n, py, px, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, py, px // 2 + 1)) + 1j * rng.standard_normal((n, py, px // 2 + 1))


@pytest.mark.parametrize("py,px", SHAPES)
def test_irfftn_matches_oracle(cuda_device, py, px):
    import torch

    from cryojax_b200 import _native as nat

    f = _half_planes(3, py, px, seed=py * 1000 + px)
    got = nat.postprocess_real(torch.as_tensor(f.astype(np.complex64)).cuda(), (py, px), (py, px))
    assert got.dtype == torch.float32 and tuple(got.shape) == (3, py, px)
    ref = np.stack([O.irfftn(x, s=(py, px)) for x in f])
    assert max(rel_l2_per_image(got.cpu().numpy(), ref)) <= IMAGE_REL_L2_TOL


@pytest.mark.parametrize("py,px,h,w", [(64, 64, 48, 40), (64, 64, 47, 41), (65, 63, 48, 40), (320, 320, 256, 255),
                                       (44, 42, 30, 30), (33, 47, 33, 20)])
@pytest.mark.parametrize("normalize", [False, True])
@pytest.mark.parametrize("with_mask", [False, True])
def test_crop_normalise_mask_matches_oracle(cuda_device, py, px, h, w, normalize, with_mask):
    import torch

    from cryojax_b200 import _native as nat

    f = _half_planes(4, py, px, seed=7 + h)
    rng = np.random.default_rng(h * w)
    mask = rng.uniform(0.0, 1.0, (h, w)) if with_mask else None
    got = nat.postprocess_real(torch.as_tensor(f.astype(np.complex64)).cuda(), (py, px), (h, w), normalize=normalize,
                               mask=None if mask is None else mask.astype(np.float32)).cpu().numpy()
    spec = O.ImageSpec(shape=(h, w), padded_shape=(py, px), pixel_size=1.0)
    ref = np.stack([O.postprocess(x, spec, normalizes_signal=normalize, mask=mask) for x in f])
    assert max(rel_l2_per_image(got, ref)) <= IMAGE_REL_L2_TOL


@pytest.mark.parametrize("py,px", SHAPES)
def test_rfft2_matches_oracle(cuda_device, py, px):
    import torch

    from cryojax_b200 import _native as nat

    x = np.random.default_rng(py + 3 * px).standard_normal((3, py, px))
    got = nat.rfft2(torch.as_tensor(x.astype(np.float32)).cuda())
    assert got.dtype == torch.complex64 and tuple(got.shape) == (3, py, px // 2 + 1)
    ref = np.stack([O.rfftn(im) for im in x])
    assert max(rel_l2_per_image(got.cpu().numpy(), ref)) <= IMAGE_REL_L2_TOL


@pytest.mark.parametrize("py,px", [(64, 64), (33, 47), (320, 320)])
def test_rfft2_inverts_irfftn(cuda_device, py, px):
    import torch

    from cryojax_b200 import _native as nat

    x = np.random.default_rng(5).standard_normal((2, py, px))
    f = np.stack([O.rfftn(im) for im in x]).astype(np.complex64)  # Hermitian where irfftn needs it
    back = nat.rfft2(nat.postprocess_real(torch.as_tensor(f).cuda(), (py, px), (py, px)))
    assert max(rel_l2_per_image(back.cpu().numpy(), f)) <= IMAGE_REL_L2_TOL


def test_many_images_take_several_passes(cuda_device):
    """A workspace for 3 images processes 10 in passes of 3 with the same result."""
    import torch

    from cryojax_b200 import _native as nat

    py, px, h, w = 40, 40, 32, 30
    f = torch.as_tensor(_half_planes(10, py, px, seed=2).astype(np.complex64)).cuda()
    one = nat.postprocess_real(f, (py, px), (h, w), normalize=True)
    ws = torch.empty(nat.postprocess_workspace_size(3, py, px), dtype=torch.uint8, device="cuda")
    three = nat.postprocess_real(f, (py, px), (h, w), normalize=True, workspace=ws)
    torch.testing.assert_close(one, three, rtol=0, atol=0)


def test_rejects_a_crop_larger_than_the_padded_shape(cuda_device):
    import torch

    from cryojax_b200 import _native as nat

    f = torch.zeros((1, 32, 17), dtype=torch.complex64, device="cuda")
    with pytest.raises(nat.CryojaxB200Error) as e:
        nat.postprocess_real(f, (32, 32), (40, 32))
    assert e.value.code == nat.CJX_ERR_INVALID_ARGUMENT


def test_simulate_real_space_launches_only_library_kernels(cuda_device):
    """simulate(outputs_real_space=True) with crop, normalisation and mask: every kernel the profiler sees is
    this library's, and the image matches the oracle's postprocess."""
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200 import simulator as S
    from cryojax_b200 import transforms as T
    from tests.helpers import make_volume, random_specs, specs_to_model_args

    vol, grid, fs = make_volume(32, 60, seed=3)
    specs = random_specs(3, seed=4, shape=(40, 36), padded_shape=(64, 64))
    pose, tt, cfg = specs_to_model_args(specs)
    dvol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
    model = S.make_image_model(dvol, cfg, pose, tt, normalizes_signal=True)
    mask = T.CustomMask(np.random.default_rng(0).uniform(0.5, 1.0, (40, 36)))
    model.simulate(mask=mask)  # warm-up
    torch.cuda.synchronize()
    with torch.profiler.profile(activities=[torch.profiler.ProfilerActivity.CUDA]) as prof:
        got = model.simulate(mask=mask)
        torch.cuda.synchronize()
    names = {e.name for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA}
    kernels = {n for n in names if not n.lower().startswith(("memcpy", "memset"))}
    assert kernels and all("cjx" in n for n in kernels), sorted(kernels)  # every kernel is in namespace cjx
    ref = np.stack([O.simulate(grid, fs, s, normalizes_signal=True, mask=mask.get()) for s in specs])
    assert max(rel_l2_per_image(got.cpu().numpy(), ref)) <= IMAGE_REL_L2_TOL
