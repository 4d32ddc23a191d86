"""GPU: the library's warp FFTs (cjx_fft_c2c, through the C-ABI) against numpy.fft in float64.

Register/shuffle form for n = 32 R, shared-memory Stockham otherwise.
Tolerance: relative L2 error <= 1e-6 per row (single-precision FFT).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [32, 64, 96, 128, 160, 192, 256, 320, 384, 512,  # register form
         24, 40, 48, 80, 83, 100, 1000, 1024]             # Stockham / direct DFT


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("direction", [-1, 1])
def test_fft_c2c_matches_numpy(cuda_device, n, direction):
    import torch

    from cryojax_b200 import _native as nat

    rng = np.random.default_rng(n)
    rows = 37
    x = (rng.standard_normal((rows, n)) + 1j * rng.standard_normal((rows, n))).astype(np.complex64)
    got = nat.fft_c2c(torch.as_tensor(x).cuda(), direction).cpu().numpy()
    xd = x.astype(np.complex128)
    ref = np.fft.fft(xd, axis=1) if direction < 0 else np.fft.ifft(xd, axis=1) * n
    err = np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert err.max() <= 1e-6, err.max()
