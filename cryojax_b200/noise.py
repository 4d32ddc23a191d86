"""Gaussian noise models on the device.

Mirror of cryoJAX's GaussianWhiteNoiseModel
(cryojax/simulator/_noise_model/gaussian_noise_model.py:128-255):
  compute_signal  scale * simulate() + offset                     (:86-110)
  compute_noise   std = sqrt(padded_n_pixels * variance) times a real
                  standard-normal half-plane with [0, 0] = 0, cast to
                  complex and post-processed like an image       (:167-205)
  sample          signal + noise                                  (:47-84)
  log_likelihood  -sum(|sim - obs|^2 / (2 var) + log(2 pi var)/2)  (:207-255)
and GaussianColoredNoiseModel (:258-397), whose per-mode variance is
padded_n_pixels * variance_fn(frequency grid) for the noise and whose
log-likelihood is evaluated in Fourier space over the rfft half plane
(mode (0, 0) dropped, the x = 0 column counted once, the rest twice).
``mask`` and ``filter`` reach the image model's simulate and, for noise,
postprocess (the filter multiplies the Fourier noise, the mask the
real-space noise).  Every quantity is per image of a batched image model;
randomness comes from a torch.Generator (JAX keys have no counterpart
here).
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

    def compute_signal(self, *, outputs_real_space=True, mask=None, filter=None):
        img = self.image_model.simulate(outputs_real_space=True, mask=mask, filter=filter)
        img = self._per_image(self.signal_scale_factor, img) * img + self._per_image(self.signal_offset, img)
        return img if outputs_real_space else _postprocess.rfftn(img)

    def _variance_grid(self, dev):
        torch = _torch()
        var = torch.as_tensor(np.asarray(self.variance, np.float64), device=dev)
        return var.reshape(-1, 1, 1) if var.dim() > 0 else var

    def compute_noise(self, generator=None, *, outputs_real_space=True, mask=None, filter=None):
        torch = _torch()
        cfg = self.image_model.image_config
        py, px = cfg.padded_shape
        n = self.image_model.batch_size
        lead = () if n is None else (n,)
        dev = self.image_model.volume_parametrization.device
        z = torch.randn(lead + (py, px // 2 + 1), generator=generator, device=dev, dtype=torch.float64)
        z[..., 0, 0] = 0.0
        f = (torch.sqrt(math.prod((py, px)) * self._variance_grid(dev)) * z).to(torch.complex64)
        if filter is not None:
            f = filter(f)
        return _postprocess.postprocess(f, cfg.shape, cfg.padded_shape, outputs_real_space=outputs_real_space,
                                        normalizes_signal=self.image_model.normalizes_signal, mask=mask)

    def sample(self, generator=None, *, outputs_real_space=True, mask=None, filter=None):
        return self.compute_signal(outputs_real_space=outputs_real_space, mask=mask, filter=filter) + \
            self.compute_noise(generator, outputs_real_space=outputs_real_space, mask=mask, filter=filter)

    def log_likelihood(self, observed, *, mask=None, filter=None):
        torch = _torch()
        sim = self.compute_signal(outputs_real_space=True, mask=mask, filter=filter).to(torch.float64)
        obs = torch.as_tensor(observed, device=sim.device, dtype=torch.float64)
        var = self._per_image(self.variance, sim)
        per_pixel = (sim - obs) ** 2 / (2 * var) + torch.log(2 * math.pi * var) / 2
        return -per_pixel.sum(dim=(-2, -1))


class GaussianColoredNoiseModel(GaussianWhiteNoiseModel):
    """Gaussian noise with a per-frequency variance.  gaussian_noise_model.py:258-397.

    ``variance_fn`` maps a (..., 2) frequency grid in 1/A to variances (a
    Constant, a FourierGaussian, or any callable); default Constant(1).
    """

    def __init__(self, image_model, variance_fn=None, signal_scale_factor=1.0, signal_offset=0.0):
        from .simulator import Constant

        if np.any(np.asarray(signal_scale_factor) <= 0):
            raise ValueError("signal_scale_factor must be positive")
        self.image_model = image_model
        self.variance_fn = variance_fn if variance_fn is not None else Constant(1.0)
        self.signal_scale_factor = signal_scale_factor
        self.signal_offset = signal_offset

    def _variance_on(self, shape, dev):
        from .transforms import make_frequency_grid

        torch = _torch()
        pixel = float(np.ravel(self.image_model.image_config.pixel_size)[0])
        v = np.broadcast_to(np.asarray(self.variance_fn(make_frequency_grid(shape, pixel)), np.float64),
                            (shape[0], shape[1] // 2 + 1))
        return torch.as_tensor(np.array(v, dtype=np.float64), device=dev)

    def _variance_grid(self, dev):
        return self._variance_on(self.image_model.image_config.padded_shape, dev)

    def log_likelihood(self, observed, *, mask=None, filter=None):
        """gaussian_noise_model.py:334-397: ``observed`` is the Fourier image ([.., H, W//2+1])."""
        torch = _torch()
        cfg = self.image_model.image_config
        n_pixels = math.prod(cfg.shape)
        sim = self.compute_signal(outputs_real_space=False, mask=mask, filter=filter).to(torch.complex128)
        obs = torch.as_tensor(observed, device=sim.device).to(torch.complex128)
        var = n_pixels * self._variance_on(cfg.shape, sim.device)
        per_mode = (sim - obs).abs() ** 2 / (2 * var) + torch.log(2 * math.pi * var) / 2
        total = per_mode[..., 1:, 0].sum(dim=-1) + 2 * per_mode[..., :, 1:].sum(dim=(-2, -1))
        return -total / n_pixels


def noise_variance_for_snr(signal_images, snr):
    """Per-image noise variance giving the requested SNR (signal variance / noise variance)."""
    torch = _torch()
    s = signal_images.to(torch.float64)
    return (s.var(dim=(-2, -1), unbiased=False) / snr).cpu().numpy()
