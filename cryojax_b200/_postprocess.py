"""Real-space postprocessing of simulated rfft images on the device.

irfftn follows cryoJAX's convention (cryojax/ndimage/_fft.py:57-77): an
inverse real FFT followed by fftshift.  Like the reference's FFT backends,
the inverse transforms the leading axis as complex and keeps only the real
part of the DC and (even size) Nyquist bins of the last axis; the columns
kx = 0 and kx = Px/2 are made Hermitian in ky first so the library C2R sees
a well-defined input.  postprocess mirrors
cryojax/simulator/_image_model/base_image_model.py:107-158 (the filter is
applied earlier, inside the device launch).
"""

from __future__ import annotations


def _hermitian_columns(f, px):
    import torch

    py = f.shape[-2]
    idx = (-torch.arange(py, device=f.device)) % py
    g = f.clone()
    cols = [0] + ([px // 2] if px % 2 == 0 else [])
    for c in cols:
        col = f[..., :, c]
        g[..., :, c] = 0.5 * (col + torch.conj(col[..., idx]))
    return g


def irfftn(fourier_image, shape):
    import torch

    py, px = shape
    f = _hermitian_columns(fourier_image, px)
    x = torch.fft.irfftn(f, s=(py, px), dim=(-2, -1))
    return torch.fft.fftshift(x, dim=(-2, -1))


def crop_to_shape(image, shape):
    """Centre crop (cryojax/ndimage/_edges.py:15-62)."""
    ny, nx = image.shape[-2:]
    h, w = shape
    yc, xc = ny // 2, nx // 2
    return image[..., yc - h // 2: yc + h // 2 + h % 2, xc - w // 2: xc + w // 2 + w % 2]


def rfftn(image):
    import torch

    return torch.fft.rfftn(torch.fft.ifftshift(image, dim=(-2, -1)), dim=(-2, -1))


def postprocess(fourier_image, shape, padded_shape, *, outputs_real_space=True, normalizes_signal=False,
                mask=None):
    if mask is None and tuple(padded_shape) == tuple(shape) and not normalizes_signal:
        return irfftn(fourier_image, shape) if outputs_real_space else fourier_image
    image = irfftn(fourier_image, padded_shape)
    if tuple(padded_shape) != tuple(shape):
        image = crop_to_shape(image, shape)
    if normalizes_signal:
        mean = image.mean(dim=(-2, -1), keepdim=True)
        std = image.std(dim=(-2, -1), keepdim=True, unbiased=False)
        image = (image - mean) / std
    if mask is not None:
        image = mask(image)
    return image if outputs_real_space else rfftn(image)
