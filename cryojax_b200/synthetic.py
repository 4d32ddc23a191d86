"""Seeded synthetic inputs with the benchmark configurations' shapes.

No public dataset is involved: volumes are sums of isotropic 3-D Gaussians
a * exp(-|r - c|^2 / (2 sigma^2)) on a box^3 voxel grid (integer voxel
coordinates [z, y, x]), each evaluated within +-5 sigma of its centre;
poses are uniform on SO(3) with uniform in-plane offsets; CTF parameters are
drawn uniformly per image.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import rotations as rot


def gaussian_sum_volume(box, n_gaussians, seed, *, centre_region=None, sigma_range=(1.0, 3.0),
                        amplitude_range=(0.5, 1.5), truncate=5.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    lo, hi = centre_region if centre_region is not None else (0.2 * box, 0.8 * box)
    centres = rng.uniform(lo, hi, size=(n_gaussians, 3))
    sigmas = rng.uniform(sigma_range[0], sigma_range[1], size=n_gaussians)
    amps = rng.uniform(amplitude_range[0], amplitude_range[1], size=n_gaussians)
    vol = np.zeros((box, box, box), np.float64)
    for c, s, a in zip(centres, sigmas, amps):
        r = int(math.ceil(truncate * s))
        base = np.floor(c).astype(int)
        lo_i = np.maximum(base - r, 0)
        hi_i = np.minimum(base + r + 1, box)
        g = [np.exp(-((np.arange(lo_i[k], hi_i[k], dtype=np.float64) - c[k]) ** 2) / (2 * s * s)) for k in range(3)]
        vol[lo_i[0]:hi_i[0], lo_i[1]:hi_i[1], lo_i[2]:hi_i[2]] += (
            a * g[0][:, None, None] * g[1][None, :, None] * g[2][None, None, :])
    return vol


@dataclass
class ImageBatch:
    wxyz: np.ndarray           # (n, 4)
    offsets: np.ndarray        # (n, 2) Angstrom
    defocus: np.ndarray        # (n,)
    astigmatism: np.ndarray    # (n,)
    astigmatism_angle: np.ndarray  # (n,) degrees


def image_batch(n, seed, *, max_offset=20.0, defocus_range=(5000.0, 25000.0), astig_range=(0.0, 500.0),
                angle_range=(0.0, 180.0)) -> ImageBatch:
    rng = np.random.default_rng(seed)
    q = rot.sample_uniform_quaternions(rng, n)
    off = rng.uniform(-max_offset, max_offset, size=(n, 2))
    return ImageBatch(q, off, rng.uniform(*defocus_range, n), rng.uniform(*astig_range, n),
                      rng.uniform(*angle_range, n))


def noisy_images(image_model, snr, generator=None):
    """Real-space images of a batched image model plus white Gaussian noise.

    SNR is signal variance / noise variance per image, in real space (the
    pose-search configurations' definition); white noise of variance s^2 in
    real space is the reference's GaussianWhiteNoiseModel draw
    (cryojax/simulator/_noise_model/gaussian_noise_model.py:167-205) up to
    its [0, 0] Fourier term.  Returns (noisy, clean) float32 CUDA tensors.
    """
    import torch

    clean = image_model.simulate(outputs_real_space=True).float()
    if clean.dim() == 2:
        clean = clean[None]
    var = clean.var(dim=(-2, -1), unbiased=False, keepdim=True) / float(snr)
    noise = torch.randn(clean.shape, generator=generator, device=clean.device, dtype=torch.float32)
    return clean + noise * torch.sqrt(var), clean
