"""Image filters and masks, and the coordinate grids they are built on.

Mirrors cryojax/ndimage/transforms/_filters.py and _masks.py and the grid
constructors of cryojax/coordinates/_make_coordinate_grids.py.  Arrays are
float64 NumPy on the host (``.array`` / ``get()``); calling a transform
multiplies an image (NumPy or torch) by it.  In an image model,
``simulate(filter=...)`` hands the filter to the device, where it is
multiplied into the Fourier image inside the simulation's epilogue
(cjx_slice_ctf_forward_filtered); masks multiply the real-space image after
the inverse transform, crop and normalisation (base_image_model.py:107-158).
"""

from __future__ import annotations

import numpy as np


def make_coordinate_grid(shape, grid_spacing=1.0):
    """(y, x, 2) real-space coordinates, [..., 0] = x, [..., 1] = y, (i - n // 2) * spacing.

    cryojax/coordinates/_make_coordinate_grids.py:100-136, 201-223, 301-317.
    """
    ny, nx = shape
    c = lambda n: (np.arange(n) - n // 2) * float(grid_spacing)
    xv, yv = np.meshgrid(c(nx), c(ny), indexing="xy")
    return np.stack([xv, yv], axis=-1)


def make_frequency_grid(shape, grid_spacing=1.0, outputs_rfftfreqs=True):
    """(y, x or x//2+1, 2) frequencies with zero in the corner, [..., 0] = kx, [..., 1] = ky.

    cryojax/coordinates/_make_coordinate_grids.py:67-97, 259-317.
    """
    ny, nx = shape
    ky = np.fft.fftfreq(ny, grid_spacing)
    kx = (np.fft.rfftfreq if outputs_rfftfreqs else np.fft.fftfreq)(nx, grid_spacing)
    xv, yv = np.meshgrid(kx, ky, indexing="xy")
    return np.stack([xv, yv], axis=-1)


def _cosine_edge(r, inner, width):
    """1 inside ``inner``, 0 beyond ``inner + width``, a raised cosine between."""
    r = np.asarray(r, np.float64)
    edge = 0.5 * (1.0 + np.cos(np.pi * (r - inner) / width)) if width > 0 else np.zeros_like(r)
    return np.where(r <= inner, 1.0, np.where(r > inner + width, 0.0, edge))


class AbstractImageTransform:
    array: np.ndarray

    def get(self):
        return self.array

    def __call__(self, image):
        try:
            import torch

            if isinstance(image, torch.Tensor):
                return image * torch.as_tensor(self.array, dtype=image.real.dtype, device=image.device)
        except ImportError:  # pragma: no cover - torch is a dependency
            pass
        return image * self.array

    def __mul__(self, other):
        return CustomFilter(self.array * other.array) if isinstance(self, AbstractFilter) else \
            CustomMask(self.array * other.array)


class AbstractFilter(AbstractImageTransform):
    """A Fourier-space multiplier over an rfft grid.  cryojax/ndimage/transforms/_filters.py:22-36."""


class CustomFilter(AbstractFilter):
    """cryojax/ndimage/transforms/_filters.py:39-55."""

    def __init__(self, filter):
        self.array = np.asarray(filter, np.float64)


class LowpassFilter(AbstractFilter):
    """Raised-cosine low-pass.  cryojax/ndimage/transforms/_filters.py:58-96, 193-226: cutoff and
    rolloff width as fractions of the Nyquist frequency 1 / (2 grid_spacing)."""

    def __init__(self, frequency_grid_in_angstroms_or_pixels, grid_spacing=1.0, frequency_cutoff_fraction=0.95,
                 rolloff_width_fraction=0.05):
        k_max = 1.0 / (2.0 * float(grid_spacing))
        k = np.linalg.norm(np.asarray(frequency_grid_in_angstroms_or_pixels, np.float64), axis=-1)
        self.array = _cosine_edge(k, frequency_cutoff_fraction * k_max, rolloff_width_fraction * k_max)


class HighpassFilter(AbstractFilter):
    """1 - LowpassFilter.  cryojax/ndimage/transforms/_filters.py:99-137."""

    def __init__(self, frequency_grid_in_angstroms_or_pixels, grid_spacing=1.0, frequency_cutoff_fraction=0.95,
                 rolloff_width_fraction=0.05):
        self.array = 1.0 - LowpassFilter(frequency_grid_in_angstroms_or_pixels, grid_spacing,
                                         frequency_cutoff_fraction, rolloff_width_fraction).array


class AbstractMask(AbstractImageTransform):
    """A real-space multiplier.  cryojax/ndimage/transforms/_masks.py:18-31."""


class CustomMask(AbstractMask):
    """cryojax/ndimage/transforms/_masks.py:34-46."""

    def __init__(self, mask_array):
        self.array = np.asarray(mask_array, np.float64)


class CircularCosineMask(AbstractMask):
    """cryojax/ndimage/transforms/_masks.py:49-81, 321-349."""

    def __init__(self, coordinate_grid, radius, rolloff_width, xy_offset=(0.0, 0.0)):
        g = np.asarray(coordinate_grid, np.float64) - np.asarray(xy_offset, np.float64)
        self.array = _cosine_edge(np.linalg.norm(g, axis=-1), float(radius), float(rolloff_width))


class SquareCosineMask(AbstractMask):
    """cryojax/ndimage/transforms/_masks.py:118-146, 352-403: soft edges per axis, multiplied in the corners."""

    def __init__(self, coordinate_grid, side_length, rolloff_width):
        g = np.abs(np.asarray(coordinate_grid, np.float64))
        s, w = float(side_length), float(rolloff_width)
        ax, ay = g[..., 0], g[..., 1]
        in_sq = lambda a, b, side: (a <= side / 2) & (b <= side / 2)
        in_edge = lambda a: (a > s / 2) & (a < s / 2 + w)
        edge = lambda a: 0.5 * (1 + np.cos(np.pi * (a - s / 2) / w))
        ex, ey = in_edge(ax), in_edge(ay)
        self.array = np.where(in_sq(ax, ay, s), 1.0,
                              np.where(in_sq(ax, ay, s + 2 * w),
                                       np.where(ex & ey, edge(ax) * edge(ay), np.where(ex, edge(ax), edge(ay))),
                                       0.0))
