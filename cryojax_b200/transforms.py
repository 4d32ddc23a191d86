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
    """Real-space coordinates (i - n // 2) * spacing: (y, x, 2) with [..., 0] = x, [..., 1] = y, or for a
    3-D shape (z, y, x, 3) with [..., 2] = z.

    cryojax/coordinates/_make_coordinate_grids.py:100-136, 201-223, 301-317.
    """
    c = lambda n: (np.arange(n) - n // 2) * float(grid_spacing)
    if len(shape) == 2:
        ny, nx = shape
        xv, yv = np.meshgrid(c(nx), c(ny), indexing="xy")
        return np.stack([xv, yv], axis=-1)
    nz, ny, nx = shape
    zv, yv, xv = np.meshgrid(c(nz), c(ny), c(nx), indexing="ij")
    return np.stack([xv, yv, zv], axis=-1)


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


class SphericalCosineMask(AbstractMask):
    """The circular mask on a 3-D coordinate grid.  cryojax/ndimage/transforms/_masks.py:84-115."""

    def __init__(self, coordinate_grid, radius, rolloff_width):
        self.array = _cosine_edge(np.linalg.norm(np.asarray(coordinate_grid, np.float64), axis=-1), float(radius),
                                  float(rolloff_width))


def _soft_box(abs_coords, widths, w):
    """A box of full widths with raised-cosine edges of width w.

    The reference's nested selection (_masks.py:352-403, 439-501, 504-583):
    1 inside the box; in the box grown by w, the product of the edge values
    of the axes whose |coordinate| lies strictly inside their edge band, or,
    when none does, the last axis's edge value; 0 beyond.
    """
    inside = np.ones(abs_coords[0].shape, bool)
    grown = np.ones(abs_coords[0].shape, bool)
    prod = np.ones(abs_coords[0].shape)
    any_edge = np.zeros(abs_coords[0].shape, bool)
    for a, s_ in zip(abs_coords, widths):
        inside &= a <= s_ / 2
        grown &= a <= s_ / 2 + w
        in_edge = (a > s_ / 2) & (a < s_ / 2 + w)
        edge = 0.5 * (1 + np.cos(np.pi * (a - s_ / 2) / w)) if w > 0 else np.zeros_like(a)
        prod = np.where(in_edge, prod * edge, prod)
        any_edge |= in_edge
    last = 0.5 * (1 + np.cos(np.pi * (abs_coords[-1] - widths[-1] / 2) / w)) if w > 0 else np.zeros_like(abs_coords[-1])
    return np.where(inside, 1.0, np.where(grown, np.where(any_edge, prod, last), 0.0))


def _rotated(coordinate_grid, angle_deg):
    g = np.asarray(coordinate_grid, np.float64)
    a = np.deg2rad(float(angle_deg))
    x, y = g[..., 0], g[..., 1]
    return x * np.cos(a) + y * np.sin(a), -x * np.sin(a) + y * np.cos(a)


class Cylindrical2DCosineMask(AbstractMask):
    """An in-plane cylinder (a band, or with ``length`` a rectangle) rotated by an angle in degrees.

    cryojax/ndimage/transforms/_masks.py:149-198, 406-501.
    """

    def __init__(self, coordinate_grid, radius, rolloff_width, in_plane_rotation_angle=0.0, length=None):
        xr, yr = _rotated(coordinate_grid, in_plane_rotation_angle)
        r, w = float(radius), float(rolloff_width)
        if length is None:
            a = np.abs(yr)
            edge = 0.5 * (1 + np.cos(np.pi * (a - r) / w)) if w > 0 else np.zeros_like(a)
            self.array = np.where(a < r, 1.0, np.where(a < r + w, edge, 0.0))
        else:
            self.array = _soft_box([np.abs(yr), np.abs(xr)], [2 * r, float(length)], w)


class Rectangular2DCosineMask(AbstractMask):
    """cryojax/ndimage/transforms/_masks.py:201-240 (the cylinder with radius y_width / 2, length x_width)."""

    def __init__(self, coordinate_grid, x_width, y_width, rolloff_width, in_plane_rotation_angle=0.0):
        xr, yr = _rotated(coordinate_grid, in_plane_rotation_angle)
        self.array = _soft_box([np.abs(yr), np.abs(xr)], [float(y_width), float(x_width)], float(rolloff_width))


class Rectangular3DCosineMask(AbstractMask):
    """cryojax/ndimage/transforms/_masks.py:243-281, 504-583."""

    def __init__(self, coordinate_grid, x_width, y_width, z_width, rolloff_width):
        g = np.abs(np.asarray(coordinate_grid, np.float64))
        self.array = _soft_box([g[..., 0], g[..., 1], g[..., 2]], [float(x_width), float(y_width), float(z_width)],
                               float(rolloff_width))


class InverseSincMask(AbstractMask):
    """1 / prod_i sinc(coordinate_i / box_i) (normalised sinc).  cryojax/ndimage/transforms/_masks.py:284-318."""

    def __init__(self, coordinate_grid_in_pixels):
        g = np.asarray(coordinate_grid_in_pixels, np.float64)
        ndim = g.ndim - 1
        box = g.shape[0:ndim][::-1]
        prod = np.ones(g.shape[:-1])
        for i in range(ndim):
            prod = prod * np.sinc(g[..., i] / box[i])
        self.array = 1.0 / prod


# ---------------------------------------------------------------------------
# Radial averages and the whitening filter
# ---------------------------------------------------------------------------


def compute_binned_radial_average(image, radial_coordinate_grid, bins):
    """Mean of ``image`` over radial bins (right-closed).  cryojax/ndimage/_radial_average.py:9-41."""
    d = np.digitize(np.asarray(radial_coordinate_grid).ravel(), bins, right=True)
    img = np.asarray(image).ravel()
    total = np.bincount(d, weights=img.real, minlength=bins.size)[: bins.size]
    if np.iscomplexobj(img):
        total = total + 1j * np.bincount(d, weights=img.imag, minlength=bins.size)[: bins.size]
    count = np.bincount(d, minlength=bins.size)[: bins.size]
    with np.errstate(invalid="ignore", divide="ignore"):
        return total / count


def interpolate_radial_average_on_grid(binned_radial_average, bins, radial_coordinate_grid,
                                       interpolation_mode="linear"):
    """cryojax/ndimage/_radial_average.py:44-88."""
    r = np.asarray(radial_coordinate_grid)
    if interpolation_mode == "nearest":
        idx = np.clip(np.digitize(r, bins, right=True), 0, bins.size - 1)
        return np.asarray(binned_radial_average)[idx]
    if interpolation_mode == "linear":
        return np.interp(r.ravel(), bins, binned_radial_average).reshape(r.shape)
    raise ValueError(f"`interpolation_mode` = {interpolation_mode} not supported. Supported interpolation modes "
                     "are 'nearest' or 'linear'.")


def make_radial_frequency_bins(shape, minimum_frequency=0.0, maximum_frequency=np.sqrt(2) / 2, pixel_size=1.0):
    """cryojax/ndimage/_fourier_statistics.py:276-280 (step 1 / max(shape))."""
    step = 1.0 / max(*shape)
    n_bins = 1 + int((maximum_frequency - minimum_frequency) / step)
    return np.linspace(minimum_frequency, maximum_frequency, n_bins) / pixel_size


def compute_binned_powerspectrum(fourier_image, radial_frequency_grid, pixel_or_voxel_size=1.0, *,
                                 minimum_frequency=0.0, maximum_frequency=np.sqrt(2) / 2):
    """cryojax/ndimage/_fourier_statistics.py:13-86."""
    power = (np.asarray(fourier_image) * np.conj(fourier_image)).real
    bins = make_radial_frequency_bins(np.shape(fourier_image), minimum_frequency, maximum_frequency,
                                      pixel_or_voxel_size)
    return compute_binned_radial_average(power, radial_frequency_grid, bins), bins


def _edge_resize(image, shape):
    """Centre crop or edge-mode pad to ``shape`` (cryojax/ndimage/_edges.py:150-185 with mode="edge")."""
    out = image
    for axis, (n, m) in enumerate(zip(image.shape, shape)):
        if m < n:
            c = n // 2
            out = np.take(out, np.arange(c - m // 2, c + m // 2 + m % 2), axis=axis)
        elif m > n:
            pad = m - n
            if m % 2 == 1 and n % 2 == 0:
                lr = (pad // 2, pad // 2 + 1)
            elif m % 2 == 0 and n % 2 == 1:
                lr = (pad // 2 + 1, pad // 2)
            else:
                lr = (pad // 2, pad // 2)
            width = [(0, 0)] * out.ndim
            width[axis] = lr
            out = np.pad(out, width, mode="edge")
    return out


class WhiteningFilter(AbstractFilter):
    """Inverse square root (or inverse) of the stack's radially averaged power spectrum.

    cryojax/ndimage/transforms/_filters.py:140-190, 229-297 (the cisTEM
    construction): power of rfft(image) / sqrt(n_pixels) binned on radial
    frequency in [0, sqrt(2)/2] with step 1 / max(rfft shape), averaged over
    the stack, interpolated back onto the grid, optionally resized to
    ``shape`` through real space (edge padding), negatives clipped, zero
    where the power is ~0, and the (0, 0) mode (and an even-even Nyquist
    corner) set to 0.
    """

    def __init__(self, image_or_image_stack, shape=None, *, interpolation_mode="linear", outputs_squared=False):
        stack = np.asarray(image_or_image_stack, np.float64)
        if stack.ndim == 2:
            stack = stack[None]
        ny, nx = stack.shape[1:]
        freqs = make_frequency_grid((ny, nx))
        radial = np.linalg.norm(freqs, axis=-1)
        fourier = np.fft.rfftn(np.fft.ifftshift(stack, axes=(1, 2)), axes=(1, 2)) / np.sqrt(ny * nx)
        spectra = []
        for f in fourier:
            p, bins = compute_binned_powerspectrum(f, radial, maximum_frequency=np.sqrt(2) / 2)
            spectra.append(p)
        power = interpolate_radial_average_on_grid(np.mean(spectra, axis=0), bins, radial, interpolation_mode)
        if shape is not None:
            real = np.fft.fftshift(np.fft.irfftn(power, s=(ny, nx), axes=(0, 1)))
            power = np.fft.rfftn(np.fft.ifftshift(_edge_resize(real, tuple(shape)))).real
            power = np.where(power < 0, 0.0, power)
            new_shape = tuple(shape)
        else:
            new_shape = (ny, nx)
        with np.errstate(divide="ignore", invalid="ignore"):
            inv = 1.0 / power if outputs_squared else 1.0 / np.sqrt(power)
        filt = np.where(np.isclose(power, 0.0), 0.0, inv)
        filt[0, 0] = 0.0
        if new_shape[0] % 2 == 0 and new_shape[1] % 2 == 0:
            filt[new_shape[0] // 2, new_shape[1] // 2] = 0.0
        self.array = filt
