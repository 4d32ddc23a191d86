"""GPU: the fused gather + column inverse FFT pass (CJX_TUNE_GATHER_MODE 2) against the oracle and the split pass.

The fused kernel samples the plane with the split gather's sampler and runs the
split column pass's transform on the same values, so with the same FFT mode the
two give bit-identical images; against the float64 oracle the tolerance is the
usual relative L2 <= 1e-5 per image.  Covered: every register-FFT volume side
from N = 32 to 512 (crop and pad), the three grid layouts, the four lane maps and
both sample counts at N = 512, both out-of-bounds rules, the Ewald sphere, and a
chunked call.
"""

import contextlib

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import IMAGE_REL_L2_TOL, make_volume, random_specs, rel_l2_per_image, specs_to_model_args

pytestmark = pytest.mark.gpu


@contextlib.contextmanager
def tuning(**kw):
    from cryojax_b200 import _native as nat

    keys = {"mode": nat.CJX_TUNE_GATHER_MODE, "ilp": nat.CJX_TUNE_GATHER_ILP, "tile": nat.CJX_TUNE_GATHER_TILE,
            "fft": nat.CJX_TUNE_FFT_MODE}
    old = {k: nat.tuning_get(keys[k]) for k in kw}
    try:
        for k, v in kw.items():
            nat.tuning_set(keys[k], v)
        yield
    finally:
        for k, v in old.items():
            nat.tuning_set(keys[k], v)


def _run(grid, specs, *, layout="pairs", ewald=False, chunk=0, oob="fill"):
    import torch

    from cryojax_b200 import simulator as S

    pose, tt, cfg = specs_to_model_args(specs)
    vol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
    cls = S.EwaldSphereExtraction if ewald else S.FourierSliceExtraction
    integ = cls(outputs_integral=False, use_bricked_layout=layout != "linear", pair_layout=layout == "pairs",
                out_of_bounds_mode=oob)
    model = S.make_image_model(vol, cfg, pose, tt, volume_integrator=integ)
    flags = model._flags() | integ._base_flags()
    out = integ.run(vol, cfg, model.image_params(), flags, images_per_chunk=chunk)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _synthetic_grid(n, seed, width=0.12):
    rng = np.random.default_rng(seed)
    k = (np.arange(n) - n // 2) / n
    env1 = np.exp(-(k**2) / (2 * width**2))
    g = (rng.standard_normal((n, n, n)) + 1j * rng.standard_normal((n, n, n))) * (
        env1[:, None, None] * env1[None, :, None] * env1[None, None, :])
    g[n // 2, n // 2, n // 2] += 50.0
    return g


# (N, image shape): every register-FFT side, crops and pads
SIZES = [(32, (16, 16)), (64, (48, 40)), (96, (64, 64)), (128, (64, 64)), (160, (96, 96)), (192, (224, 200)),
         (256, (128, 128)), (320, (192, 192)), (384, (192, 192)), (512, (320, 320))]


@pytest.mark.parametrize("n,shape", SIZES)
def test_fused_pass_matches_oracle_and_split_pass(cuda_device, n, shape):
    grid = _synthetic_grid(n, seed=n + 3)
    fs = O.make_frequency_slice((n, n), outputs_rfftfreqs=False)
    specs = random_specs(3, seed=n + 4, shape=shape)
    with tuning(mode=2):
        fused = _run(grid, specs)
    with tuning(mode=1):
        split = _run(grid, specs)
    np.testing.assert_array_equal(fused, split)
    ref = np.stack([O.compute_fourier_image(grid, fs, s) for s in specs])
    errs = rel_l2_per_image(fused, ref)
    assert max(errs) <= IMAGE_REL_L2_TOL, errs


@pytest.mark.parametrize("ilp,tile", [(1, 0), (1, 1), (1, 2), (1, 3), (2, 0), (2, 1), (2, 2), (2, 3), (4, 1)])
def test_fused_lane_maps_and_sample_counts(cuda_device, ilp, tile):
    n, shape = 512, (320, 320)
    grid = _synthetic_grid(n, seed=91)
    specs = random_specs(2, seed=92, shape=shape)
    with tuning(mode=1):
        split = _run(grid, specs)
    with tuning(mode=2, ilp=ilp, tile=tile):
        fused = _run(grid, specs)
    np.testing.assert_array_equal(fused, split)


@pytest.mark.parametrize("layout", ["pairs", "bricked", "linear"])
@pytest.mark.parametrize("fft", [1, 2])
def test_fused_layouts_and_fft_modes(cuda_device, layout, fft):
    vol, grid, fs = make_volume(64, 120, seed=5)  # N = 128: every face is reached by some samples
    specs = random_specs(4, seed=6, shape=(96, 80))
    with tuning(mode=2, fft=fft):
        fused = _run(grid, specs, layout=layout)
    ref = np.stack([O.compute_fourier_image(grid, fs, s) for s in specs])
    assert max(rel_l2_per_image(fused, ref)) <= IMAGE_REL_L2_TOL


@pytest.mark.parametrize("oob", ["fill", "zero_fill_negative"])
def test_fused_out_of_bounds_rules(cuda_device, oob):
    vol, grid, fs = make_volume(32, 60, seed=8)
    specs = random_specs(4, seed=9, shape=(32, 32))
    with tuning(mode=2):
        fused = _run(grid, specs, oob=oob)
    ref = np.stack([O.compute_fourier_image(grid, fs, s, wrap_negative=(oob == "fill")) for s in specs])
    assert max(rel_l2_per_image(fused, ref)) <= IMAGE_REL_L2_TOL


def test_fused_ewald_sphere(cuda_device):
    vol, grid, fs = make_volume(48, 100, seed=12)  # N = 96
    specs = random_specs(3, seed=13, shape=(64, 64))
    with tuning(mode=2):
        fused = _run(grid, specs, ewald=True)
    with tuning(mode=1):
        split = _run(grid, specs, ewald=True)
    np.testing.assert_array_equal(fused, split)
    ref = np.stack([O.compute_fourier_image(grid, fs, s, ewald=True) for s in specs])
    assert max(rel_l2_per_image(fused, ref)) <= IMAGE_REL_L2_TOL


def test_fused_chunked_call(cuda_device):
    vol, grid, fs = make_volume(32, 60, seed=21)
    specs = random_specs(11, seed=22, shape=(40, 40))
    with tuning(mode=2):
        one = _run(grid, specs)
        chunked = _run(grid, specs, chunk=3)
    np.testing.assert_array_equal(one, chunked)
    ref = np.stack([O.compute_fourier_image(grid, fs, s) for s in specs])
    assert max(rel_l2_per_image(chunked, ref)) <= IMAGE_REL_L2_TOL
