"""Real-space output and post-processing of simulated rfft images, on this library's kernels.

irfftn follows cryoJAX's convention (cryojax/ndimage/_fft.py:57-77): an
inverse real FFT of the rfft half plane followed by fftshift; rfftn is
ifftshift then rfft2 (cryojax/ndimage/_fft.py:80-99).  postprocess mirrors
cryojax/simulator/_image_model/base_image_model.py:107-158: irfftn -> centre
crop -> normalise -> mask, in one cjx_postprocess_real call (the Fourier
filter is applied earlier, inside the simulation launch).  Masks that are
cryoJAX transform objects (or arrays) are multiplied in inside that call; any
other callable is applied to its output.
"""

from __future__ import annotations

from . import _native as nat


def irfftn(fourier_image, shape):
    """float32 real-space images [..., Py, Px] of complex64 rfft half planes [..., Py, Px//2+1]."""
    return nat.postprocess_real(fourier_image, shape, shape)


def crop_to_shape(image, shape):
    """Centre crop (cryojax/ndimage/_edges.py:15-62) of a real-space array (a view)."""
    ny, nx = image.shape[-2:]
    h, w = shape
    yc, xc = ny // 2, nx // 2
    return image[..., yc - h // 2: yc + h // 2 + h % 2, xc - w // 2: xc + w // 2 + w % 2]


def rfftn(image):
    """complex64 rfft half planes [..., Py, Px//2+1] of float real-space images [..., Py, Px]."""
    return nat.rfft2(image)


def _mask_array(mask):
    """The real-space array of a mask object (AbstractMask.get()) or array; None for other callables."""
    if mask is None:
        return None
    if hasattr(mask, "get"):
        return mask.get()
    if callable(mask):
        return None
    return mask


def postprocess(fourier_image, shape, padded_shape, *, outputs_real_space=True, normalizes_signal=False,
                mask=None):
    if mask is None and tuple(padded_shape) == tuple(shape) and not normalizes_signal:
        return irfftn(fourier_image, shape) if outputs_real_space else fourier_image
    arr = _mask_array(mask)
    image = nat.postprocess_real(fourier_image, padded_shape, shape, normalize=normalizes_signal, mask=arr)
    if mask is not None and arr is None:
        image = mask(image)
    return image if outputs_real_space else rfftn(image)
