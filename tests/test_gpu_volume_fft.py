"""GPU: the volume preparation's 3-D FFT on the library's kernels against torch.fft in float64.

FourierVoxelGridVolume.from_real_voxel_grid runs pad -> ifftshift -> fftn ->
fftshift with the batched warp FFTs (one pass per axis).  Tolerance: every
entry within 2e-6 of the largest (single-precision transforms with
double-precision twiddles against float64), for power-of-two, mixed-radix,
prime (direct DFT) and odd sides, and the benchmark's N = 512.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("box,pad", [(32, 2.0), (48, 2.0), (64, 1.3), (25, 1.0), (256, 2.0)])
def test_native_volume_fft_matches_float64(cuda_device, box, pad):
    import time

    import torch

    from cryojax_b200 import simulator as S
    from cryojax_b200 import synthetic

    vol = torch.as_tensor(synthetic.gaussian_sum_volume(box, 200, box), device="cuda")
    times = {}
    grids = {}
    for backend in ("native", "torch"):
        S.FourierVoxelGridVolume.from_real_voxel_grid(vol, pad_scale=pad, fft_backend=backend)  # warm-up
        torch.cuda.synchronize()
        t = time.perf_counter()
        grids[backend] = S.FourierVoxelGridVolume.from_real_voxel_grid(vol, pad_scale=pad,
                                                                       fft_backend=backend).fourier_voxel_grid
        torch.cuda.synchronize()
        times[backend] = time.perf_counter() - t
    a, b = grids["native"], grids["torch"]
    assert a.shape == b.shape == (int(box * pad),) * 3
    err = ((a - b).abs().max() / b.abs().max()).item()
    print(f"N={a.shape[0]} max rel err {err:.2e}; native {times['native'] * 1e3:.1f} ms, "
          f"torch float64 {times['torch'] * 1e3:.1f} ms")
    assert err <= 2e-6, err
