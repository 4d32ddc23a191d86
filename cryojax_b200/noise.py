"""Gaussian white noise model on the device.

Mirror of cryoJAX's GaussianWhiteNoiseModel
(cryojax/simulator/_noise_model/gaussian_noise_model.py:128-255):
  compute_signal  scale * simulate() + offset                     (:86-110)
  compute_noise   std = sqrt(padded_n_pixels * variance) times a real
                  standard-normal half-plane with [0, 0] = 0, cast to
                  complex and post-processed like an image       (:167-205)
  sample          signal + noise                                  (:47-84)
  log_likelihood  -sum(|sim - obs|^2 / (2 var) + log(2 pi var)/2)  (:207-255)
Every quantity is per image of a batched image model; randomness comes from
a torch.Generator (JAX keys have no counterpart here).
"""

from __future__ import annotations

import math

import numpy as np

from . import _postprocess


def _torch():
    import torch

    return torch


class GaussianWhiteNoiseModel:
    def __init__(self, image_model, variance=1.0, signal_scale_factor=1.0, signal_offset=0.0):
        if np.any(np.asarray(variance) <= 0) or np.any(np.asarray(signal_scale_factor) <= 0):
            raise ValueError("variance and signal_scale_factor must be positive")
        self.image_model = image_model
        self.variance = variance
        self.signal_scale_factor = signal_scale_factor
        self.signal_offset = signal_offset

    def _per_image(self, x, like):
        torch = _torch()
        t = torch.as_tensor(np.asarray(x, np.float64), device=like.device, dtype=like.dtype)
        return t.reshape(-1, *([1] * (like.dim() - 1))) if t.dim() > 0 and like.dim() > 2 else t

    def compute_signal(self, *, outputs_real_space=True):
        img = self.image_model.simulate(outputs_real_space=True)
        img = self._per_image(self.signal_scale_factor, img) * img + self._per_image(self.signal_offset, img)
        return img if outputs_real_space else _postprocess.rfftn(img)

    def compute_noise(self, generator=None, *, outputs_real_space=True):
        torch = _torch()
        cfg = self.image_model.image_config
        py, px = cfg.padded_shape
        n = self.image_model.batch_size
        lead = () if n is None else (n,)
        dev = self.image_model.volume_parametrization.device
        z = torch.randn(lead + (py, px // 2 + 1), generator=generator, device=dev, dtype=torch.float64)
        z[..., 0, 0] = 0.0
        var = torch.as_tensor(np.asarray(self.variance, np.float64), device=dev)
        if var.dim() > 0:
            var = var.reshape(-1, 1, 1)
        f = (torch.sqrt(math.prod((py, px)) * var) * z).to(torch.complex64)
        return _postprocess.postprocess(f, cfg.shape, cfg.padded_shape, outputs_real_space=outputs_real_space)

    def sample(self, generator=None, *, outputs_real_space=True):
        return self.compute_signal(outputs_real_space=outputs_real_space) + self.compute_noise(
            generator, outputs_real_space=outputs_real_space)

    def log_likelihood(self, observed):
        torch = _torch()
        sim = self.compute_signal(outputs_real_space=True).to(torch.float64)
        obs = torch.as_tensor(observed, device=sim.device, dtype=torch.float64)
        var = self._per_image(self.variance, sim)
        per_pixel = (sim - obs) ** 2 / (2 * var) + torch.log(2 * math.pi * var) / 2
        return -per_pixel.sum(dim=(-2, -1))


def noise_variance_for_snr(signal_images, snr):
    """Per-image noise variance giving the requested SNR (signal variance / noise variance)."""
    torch = _torch()
    s = signal_images.to(torch.float64)
    return (s.var(dim=(-2, -1), unbiased=False) / snr).cpu().numpy()
