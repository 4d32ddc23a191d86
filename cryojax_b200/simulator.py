"""Host-side mirror of cryoJAX's simulator API for the Fourier-slice path.

Same class names, argument names and meanings as ``cryojax.simulator``
(the reference is JAX/Equinox; this mirror holds NumPy parameters on the
host and torch CUDA tensors on the device).  Every field of a pose, CTF or
image config may carry a leading batch axis: a batched model simulates all
its images in ONE launch of ``cjx_slice_ctf_forward`` — the counterpart of
wrapping ``simulate`` in ``eqx.filter_vmap`` over (pose, transfer theory)
with the volume broadcast.

Covered (reference file:line):
  BasicImageConfig            cryojax/simulator/_image_config.py:280-338
  EulerAnglePose, QuaternionPose, AxisAnglePose
                              cryojax/simulator/_pose.py:203-403
  AstigmaticCTF               cryojax/simulator/_transfer_theory/transfer_function.py:84-169
  ContrastTransferTheory      cryojax/simulator/_transfer_theory/transfer_theory.py:21-119
  FourierGaussian (envelope)  cryojax/ndimage/operators/_fourier_operator.py:183-234
  Constant (envelope)         cryojax/ndimage/operators/_base_operator.py:53-67
  GaussianMixtureVolume       cryojax/simulator/_volume/representations/gaussian_volume.py:21-204
  GaussianMixtureRenderFn     cryojax/simulator/_volume_rendering/gaussian_rendering.py:24-336
  FourierVoxelGridVolume      cryojax/simulator/_volume/representations/voxel_volume.py:40-119
  FourierVoxelSplineVolume    cryojax/simulator/_volume/representations/voxel_volume.py:122-203
  FourierSliceExtraction      cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:26-183
  EwaldSphereExtraction       cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:225-516
  WeakPhaseScatteringTheory   cryojax/simulator/_scattering_theory/weak_phase_scattering_theory.py:13-80
  LinearImageModel, ProjectionImageModel
                              cryojax/simulator/_image_model/base_image_model.py:216-432
  ContrastImageModel          cryojax/simulator/_image_model/physical_image_model.py:30-137
  make_image_model            cryojax/simulator/_api_utils.py:36-223
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from . import _native as nat
from . import constants as C
from . import rotations as rot

# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------


def _arr(x):
    return np.asarray(x, dtype=np.float64)


def _batch_size(*xs) -> int | None:
    """Size of the common leading batch axis (None if all are unbatched)."""
    n = None
    for x in xs:
        if x is None:
            continue
        a = np.asarray(x)
        if a.ndim == 0:
            continue
        if n is None:
            n = a.shape[0]
        elif a.shape[0] != n and a.shape[0] != 1:
            raise ValueError(f"inconsistent batch sizes {n} and {a.shape[0]}")
    return n


def _per_image(x, n):
    a = _arr(x)
    if a.ndim == 0:
        return np.full(n, float(a))
    return np.broadcast_to(a.reshape(a.shape[0]), (n,)).astype(np.float64)


def _require_positive(name, x):
    if np.any(_arr(x) <= 0):
        raise ValueError(f"`{name}` must be positive")


# ---------------------------------------------------------------------------
# Image configuration
# ---------------------------------------------------------------------------


class BasicImageConfig:
    """Image shape, pixel size, voltage and padding options.

    cryojax/simulator/_image_config.py:280-338 (``pad_options`` keys
    ``shape`` and ``mode``; only ``mode="constant"`` is implemented on the
    device).
    """

    def __init__(self, shape, pixel_size, voltage_in_kilovolts, *, pad_options: dict | None = None):
        pad_options = dict(pad_options or {})
        self.shape = tuple(int(s) for s in shape)
        _require_positive("pixel_size", pixel_size)
        _require_positive("voltage_in_kilovolts", voltage_in_kilovolts)
        self.pixel_size = _arr(pixel_size)
        self.voltage_in_kilovolts = _arr(voltage_in_kilovolts)
        self.pad_options = {
            "shape": tuple(int(s) for s in pad_options.get("shape", self.shape)),
            "mode": pad_options.get("mode", "constant"),
        }
        if self.padded_shape[0] < self.shape[0] or self.padded_shape[1] < self.shape[1]:
            raise AttributeError("`padded_shape` is less than `shape` in one or more dimensions.")

    @property
    def padded_shape(self):
        return self.pad_options["shape"]

    @property
    def pad_mode(self):
        return self.pad_options["mode"]

    @property
    def wavelength_in_angstroms(self):
        return C.wavelength_from_kilovolts(self.voltage_in_kilovolts)

    @property
    def interaction_constant(self):
        return C.interaction_constant_from_kilovolts(self.voltage_in_kilovolts)

    @property
    def n_pixels(self):
        return math.prod(self.shape)

    @property
    def padded_n_pixels(self):
        return math.prod(self.padded_shape)


# ---------------------------------------------------------------------------
# Poses
# ---------------------------------------------------------------------------


class AbstractPose:
    offset_in_angstroms: np.ndarray

    def rotation_matrices(self) -> np.ndarray:
        """(..., 3, 3) float64 matrices R with rotated k = R k."""
        return rot.quat_to_matrix(self.quaternion())

    def quaternion(self) -> np.ndarray:  # pragma: no cover - abstract
        raise NotImplementedError

    @property
    def offset_z_in_angstroms(self):
        o = self.offset_in_angstroms
        return None if o.shape[-1] == 2 else o[..., 2]

    @property
    def batch_size(self):
        q = self.quaternion()
        return None if q.ndim == 1 else q.shape[0]


def _stack_offsets(x, y, z):
    arrs = [_arr(x), _arr(y)] + ([] if z is None else [_arr(z)])
    arrs = np.broadcast_arrays(*arrs)
    return np.stack(arrs, axis=-1)


class EulerAnglePose(AbstractPose):
    """zyz extrinsic Euler angles in degrees.  cryojax/simulator/_pose.py:203-280."""

    def __init__(self, offset_x_in_angstroms=0.0, offset_y_in_angstroms=0.0, phi_angle=0.0,
                 theta_angle=0.0, psi_angle=0.0, *, offset_z_in_angstroms=None):
        self.offset_in_angstroms = _stack_offsets(offset_x_in_angstroms, offset_y_in_angstroms, offset_z_in_angstroms)
        self.phi_angle = _arr(phi_angle)
        self.theta_angle = _arr(theta_angle)
        self.psi_angle = _arr(psi_angle)

    def quaternion(self):
        return rot.euler_zyz_to_quat(self.phi_angle, self.theta_angle, self.psi_angle)


class QuaternionPose(AbstractPose):
    """Unit quaternion q / |q|.  cryojax/simulator/_pose.py:283-335."""

    def __init__(self, offset_x_in_angstroms=0.0, offset_y_in_angstroms=0.0, wxyz=(1.0, 0.0, 0.0, 0.0), *,
                 offset_z_in_angstroms=None):
        self.offset_in_angstroms = _stack_offsets(offset_x_in_angstroms, offset_y_in_angstroms, offset_z_in_angstroms)
        wxyz = _arr(wxyz)
        if wxyz.shape[-1] != 4:
            raise ValueError("Expected `wxyz` to be a sequence of floats with length 4")
        self.wxyz = wxyz

    def quaternion(self):
        return rot.quat_normalize(self.wxyz)


class AxisAnglePose(AbstractPose):
    """Euler vector in degrees through the exponential map.  cryojax/simulator/_pose.py:338-403."""

    def __init__(self, offset_x_in_angstroms=0.0, offset_y_in_angstroms=0.0, euler_vector=(0.0, 0.0, 0.0), *,
                 offset_z_in_angstroms=None):
        self.offset_in_angstroms = _stack_offsets(offset_x_in_angstroms, offset_y_in_angstroms, offset_z_in_angstroms)
        ev = _arr(euler_vector)
        if ev.shape[-1] != 3:
            raise ValueError("Expected `euler_vector` to be a sequence of floats with length 3")
        self.euler_vector = ev

    def quaternion(self):
        return rot.so3_exp(np.deg2rad(self.euler_vector))


# ---------------------------------------------------------------------------
# CTF, envelope, transfer theory
# ---------------------------------------------------------------------------


class AstigmaticCTF:
    """cryojax/simulator/_transfer_theory/transfer_function.py:84-169."""

    def __init__(self, defocus_in_angstroms=10000.0, astigmatism_in_angstroms=0.0, astigmatism_angle=0.0,
                 spherical_aberration_in_mm=2.7):
        if np.any(_arr(spherical_aberration_in_mm) < 0):
            raise ValueError("`spherical_aberration_in_mm` must be non-negative")
        self.defocus_in_angstroms = _arr(defocus_in_angstroms)
        self.astigmatism_in_angstroms = _arr(astigmatism_in_angstroms)
        self.astigmatism_angle = _arr(astigmatism_angle)
        self.spherical_aberration_in_mm = _arr(spherical_aberration_in_mm)


class FourierGaussian:
    """amplitude * exp(-b_factor k^2 / 4).  cryojax/ndimage/operators/_fourier_operator.py:183-234."""

    def __init__(self, amplitude=1.0, b_factor=1.0):
        _require_positive("b_factor", b_factor)
        self.amplitude = _arr(amplitude)
        self.b_factor = _arr(b_factor)

    def __call__(self, frequency_grid):
        """amplitude * exp(-b |k|^2 / 4) on a (..., 2) frequency grid (cycles / A)."""
        k2 = np.sum(np.square(np.asarray(frequency_grid, np.float64)), axis=-1)
        return self.amplitude * np.exp(-0.25 * self.b_factor * k2)


class Constant:
    """A constant envelope (RELION's scale factor alone).  cryojax/ndimage/operators/_base_operator.py:53-67."""

    def __init__(self, value):
        self.value = _arr(value)

    def __call__(self, frequency_grid=None, *args, **kwargs):
        return self.value


def _envelope_amp_b(envelope):
    """(amplitude, b_factor) of a device envelope: a Constant is amplitude * exp(-0 k^2 / 4)."""
    if isinstance(envelope, Constant):
        return envelope.value, np.zeros_like(envelope.value)
    return envelope.amplitude, envelope.b_factor


class ContrastTransferTheory:
    """cryojax/simulator/_transfer_theory/transfer_theory.py:21-119 (projection branch)."""

    def __init__(self, ctf: AstigmaticCTF, envelope: FourierGaussian | Constant | None = None,
                 amplitude_contrast_ratio=0.1, phase_shift=0.0):
        ac = _arr(amplitude_contrast_ratio)
        if np.any(ac < 0) or np.any(ac > 1):
            raise ValueError("`amplitude_contrast_ratio` must be in [0, 1]")
        if envelope is not None and not isinstance(envelope, (FourierGaussian, Constant)):
            raise NotImplementedError("only FourierGaussian and Constant envelopes run on the device")
        self.ctf = ctf
        self.envelope = envelope
        self.amplitude_contrast_ratio = ac
        self.phase_shift = _arr(phase_shift)


# ---------------------------------------------------------------------------
# Volume
# ---------------------------------------------------------------------------


def _torch():
    import torch

    return torch


def fftn_native(x):
    """numpy.fft.fftn of a complex64 CUDA tensor [nz, ny, nx] with the library's batched warp FFTs
    (cjx_fft_c2c): one pass per axis, that axis moved last (one contiguous copy) for its pass."""
    for axis in (2, 1, 0):
        x = nat.fft_c2c(x.movedim(axis, -1).contiguous(), -1).movedim(-1, axis)
    return x.contiguous()


def _centred_fourier_grid(real_voxel_grid, pad_scale, pad_mode, device, fft_dtype, fft_backend="native"):
    """pad -> ifftshift -> fftn -> fftshift, complex64 on ``device``
    (cryojax/simulator/_volume/representations/voxel_volume.py:69-119, 163-203).

    ``fft_backend="native"``: the 3-D transform runs on this library's FFT
    kernels in single precision; ``"torch"``: torch.fft in ``fft_dtype``
    (float64 by default), for comparison.
    """
    torch = _torch()
    if pad_scale < 1.0:
        raise ValueError("`pad_scale` must be greater than 1.0")
    if pad_mode != "constant":
        raise NotImplementedError("only constant padding is implemented")
    real = real_voxel_grid
    if not isinstance(real, torch.Tensor):
        real = torch.as_tensor(np.asarray(real, np.float64))
    real = real.to(device=device, dtype=fft_dtype or torch.float64)
    shape = tuple(int(s * pad_scale) for s in real.shape)
    pads = []
    for s, d in zip(reversed(shape), reversed(real.shape)):
        pad = s - d
        if s % 2 == 1 and d % 2 == 0:
            lr = (pad // 2, pad // 2 + 1)
        elif s % 2 == 0 and d % 2 == 1:
            lr = (pad // 2 + 1, pad // 2)
        else:
            lr = (pad // 2, pad // 2)
        pads.extend(lr)
    padded = torch.nn.functional.pad(real, pads, mode="constant", value=0.0)
    if fft_backend == "native":
        ft = fftn_native(torch.fft.ifftshift(padded).to(torch.complex64))
        return torch.fft.fftshift(ft).contiguous()
    if fft_backend != "torch":
        raise ValueError("fft_backend must be 'native' or 'torch'")
    ft = torch.fft.fftn(torch.fft.ifftshift(padded))
    return torch.fft.fftshift(ft).to(torch.complex64).contiguous()


class FourierVoxelGridVolume:
    """Centred full 3-D FFT grid of a padded real volume (complex64, CUDA).

    cryojax/simulator/_volume/representations/voxel_volume.py:40-119.  The
    kernels read the grid as stored (C-order [z][y][x], zero frequency at
    index N//2); ``frequency_slice_in_pixels`` is implicit (the rotated plane
    is generated in the kernel from the pose).
    """

    def __init__(self, fourier_voxel_grid, rotation=None, *, bricked=None, pairs=None):
        torch = _torch()
        g = fourier_voxel_grid
        if not isinstance(g, torch.Tensor):
            g = torch.as_tensor(np.asarray(g))
        if g.dim() != 3 or len(set(g.shape)) != 1:
            raise AttributeError("Only cubic boxes are supported for fourier slice extraction.")
        self.fourier_voxel_grid = g.contiguous()  # the kernels read C order
        self.rotation = rotation  # AbstractPose attached by rotate_to_pose
        self._bricked = bricked   # device re-layouts for the gather (built on first use)
        self._pairs = pairs

    def bricked_grid(self):
        """The grid in the library's bricked layout (cached; same values)."""
        if self._bricked is None:
            self._bricked = nat.brick_volume(self.fourier_voxel_grid.contiguous())
        return self._bricked

    def pair_grid(self):
        """The grid in the x-pair bricked layout (cached; twice the grid's bytes)."""
        if self._pairs is None:
            self._pairs = nat.brick_volume_pairs_new(self.fourier_voxel_grid.contiguous())
        return self._pairs

    @property
    def shape(self):
        return tuple(self.fourier_voxel_grid.shape)

    @property
    def device(self):
        return self.fourier_voxel_grid.device

    @classmethod
    def from_real_voxel_grid(cls, real_voxel_grid, *, pad_scale: float = 1.0, pad_mode: str = "constant",
                             device: str = "cuda", fft_dtype=None, fft_backend: str = "native"):
        """pad -> ifftshift -> fftn -> fftshift, as the reference (voxel_volume.py:69-119).

        The 3-D FFT runs on ``device`` with this library's FFT kernels
        (``fft_backend="torch"``: torch.fft in float64) and the grid is stored
        as complex64 (one-time volume preparation).
        """
        return cls(_centred_fourier_grid(real_voxel_grid, pad_scale, pad_mode, device, fft_dtype, fft_backend))

    def rotate_to_pose(self, pose: AbstractPose, inverse: bool = False):
        """Attach the pose (the frequency slice is rotated inside the kernel)."""
        if inverse:
            pose = QuaternionPose(*np.moveaxis(pose.offset_in_angstroms[..., :2], -1, 0),
                                  wxyz=rot.quat_inverse(pose.quaternion()))
        return FourierVoxelGridVolume(self.fourier_voxel_grid, rotation=pose, bricked=self._bricked,
                                      pairs=self._pairs)

    def get_representation(self, rng_key=None):
        return self


class FourierVoxelSplineVolume:
    """Cubic-spline coefficients ((N+2)^3 complex64, CUDA) of a centred
    Fourier voxel grid.

    cryojax/simulator/_volume/representations/voxel_volume.py:122-203.  The
    slice is cubic-spline interpolated from the coefficients
    (fourier_voxel_extract.py:148-183); ``shape`` is the voxel grid's.
    """

    def __init__(self, spline_coefficients, rotation=None, *, bricked=None, pairs=None):
        torch = _torch()
        c = spline_coefficients
        if not isinstance(c, torch.Tensor):
            c = torch.as_tensor(np.asarray(c))
        if c.dim() != 3 or len(set(c.shape)) != 1:
            raise AttributeError("Only cubic boxes are supported for fourier slice extraction.")
        self.spline_coefficients = c.contiguous()  # the kernels read C order
        self.rotation = rotation
        self._bricked = bricked
        self._pairs = pairs

    def bricked_grid(self):
        """The coefficients in the library's bricked layout on side N + 2 (cached)."""
        if self._bricked is None:
            self._bricked = nat.brick_volume(self.spline_coefficients.contiguous())
        return self._bricked

    def pair_grid(self):
        """The coefficients in the x-pair bricked layout on side N + 2 (cached; twice their bytes)."""
        if self._pairs is None:
            self._pairs = nat.brick_volume_pairs_new(self.spline_coefficients.contiguous())
        return self._pairs

    @property
    def shape(self):
        return tuple(s - 2 for s in self.spline_coefficients.shape)

    @property
    def device(self):
        return self.spline_coefficients.device

    @classmethod
    def from_real_voxel_grid(cls, real_voxel_grid, *, pad_scale: float = 1.0, pad_mode: str = "constant",
                             device: str = "cuda", fft_dtype=None, fft_backend: str = "native"):
        """Fourier grid as FourierVoxelGridVolume.from_real_voxel_grid, then its
        spline coefficients on the device (voxel_volume.py:163-203)."""
        grid = _centred_fourier_grid(real_voxel_grid, pad_scale, pad_mode, device, fft_dtype, fft_backend)
        return cls(nat.spline_coefficients(grid))

    @classmethod
    def from_fourier_voxel_grid(cls, volume: FourierVoxelGridVolume):
        """Spline coefficients of an existing FourierVoxelGridVolume's grid."""
        return cls(nat.spline_coefficients(volume.fourier_voxel_grid.contiguous()))

    def rotate_to_pose(self, pose: AbstractPose, inverse: bool = False):
        """Attach the pose (the frequency slice is rotated inside the kernel)."""
        if inverse:
            pose = QuaternionPose(*np.moveaxis(pose.offset_in_angstroms[..., :2], -1, 0),
                                  wxyz=rot.quat_inverse(pose.quaternion()))
        return FourierVoxelSplineVolume(self.spline_coefficients, rotation=pose, bricked=self._bricked,
                                        pairs=self._pairs)

    def get_representation(self, rng_key=None):
        return self


class GaussianMixtureVolume:
    """Atoms as mixtures of isotropic Gaussians.

    cryojax/simulator/_volume/representations/gaussian_volume.py:21-204:
    ``positions`` [n, 3] (Angstrom), ``amplitudes`` and ``variances``
    (Angstrom^2) scalars, [n] or [n, n_gaussians], broadcast to
    [n, n_gaussians]; variances must be positive.  Rendered to a voxel grid
    on the device by GaussianMixtureRenderFn.
    """

    def __init__(self, positions, amplitudes=1.0, variances=1.0):
        pos = np.asarray(positions, np.float64)
        if pos.ndim != 2 or pos.shape[1] != 3:
            raise ValueError("`positions` must have shape (n_positions, 3)")
        n = pos.shape[0]

        def as_2d(name, v):
            v = np.asarray(v, np.float64)
            if v.ndim == 0:
                v = v[None, None]
            elif v.ndim == 1:
                v = v[:, None]
            elif v.ndim != 2:
                raise ValueError(f"`{name}` must be of shape (), (n_positions,) or (n_positions, n_gaussians)")
            return v

        amp, var = as_2d("amplitudes", amplitudes), as_2d("variances", variances)
        g = max(amp.shape[1], var.shape[1])
        self.positions = pos
        self.amplitudes = np.broadcast_to(amp, (n, g)).copy()
        self.variances = np.broadcast_to(var, (n, g)).copy()
        if np.any(self.variances <= 0):
            raise ValueError("`variances` must be positive")

    @classmethod
    def from_tabulated_parameters(cls, atom_positions, parameters, extra_b_factors=None):
        """gaussian_volume.py:144-183: amplitudes a, variances (b + extra B) / (8 pi^2) (Peng et al. 1996)."""
        a = np.asarray(parameters.a if hasattr(parameters, "a") else parameters["a"], np.float64)
        b = np.asarray(parameters.b if hasattr(parameters, "b") else parameters["b"], np.float64)
        if extra_b_factors is not None:
            extra = np.asarray(extra_b_factors, np.float64)
            b = b + (extra[:, None] if extra.ndim == 1 else extra)
        return cls(atom_positions, a, C.b_factor_to_variance(b))

    def rotate_to_pose(self, pose: AbstractPose, inverse: bool = False):
        """gaussian_volume.py:185-192: positions rotated by the pose's rotation (or its inverse)."""
        R = pose.rotation_matrices()
        if R.ndim != 2:
            raise ValueError("rotate a GaussianMixtureVolume with one pose at a time")
        if inverse:
            R = R.T
        return GaussianMixtureVolume(self.positions @ R.T, self.amplitudes, self.variances)

    def translate_to_pose(self, pose: AbstractPose):
        """gaussian_volume.py:194-204."""
        o = np.asarray(pose.offset_in_angstroms, np.float64)
        if o.ndim != 1:
            raise ValueError("translate a GaussianMixtureVolume with one pose at a time")
        if o.shape[0] == 2:
            o = np.concatenate([o, [0.0]])
        return GaussianMixtureVolume(self.positions + o, self.amplitudes, self.variances)


class GaussianMixtureRenderFn:
    """Render a GaussianMixtureVolume to a voxel grid on the device.

    cryojax/simulator/_volume_rendering/gaussian_rendering.py:24-197: the
    voxel-averaged potential (error-function integrals per axis), here
    splatted atom by atom (cjx_render_gaussians).  ``batch_options`` are
    accepted for API compatibility and have no effect (the device kernel
    needs no batching over z-planes or atoms).
    """

    def __init__(self, shape, voxel_size, *, batch_options: dict | None = None):
        self.shape = tuple(int(s) for s in shape)
        if len(self.shape) != 3:
            raise ValueError("`shape` must be (z_dim, y_dim, x_dim)")
        _require_positive("voxel_size", voxel_size)
        self.voxel_size = float(voxel_size)
        self.batch_options = dict(batch_options or {})

    def __call__(self, volume_representation: GaussianMixtureVolume, *, outputs_real_space: bool = True,
                 outputs_rfft: bool = False, fftshifted: bool = False, device: str = "cuda"):
        torch = _torch()
        v = volume_representation
        if v.amplitudes.shape[1] > nat.CJX_RENDER_MAX_GAUSSIANS:
            raise NotImplementedError(f"at most {nat.CJX_RENDER_MAX_GAUSSIANS} Gaussians per position")
        t = lambda a: torch.as_tensor(a, dtype=torch.float32, device=device)
        real = nat.render_gaussians(self.shape, self.voxel_size, t(v.positions), t(v.amplitudes), t(v.variances))
        if outputs_real_space:
            return real
        # cryojax.ndimage fftn / rfftn transform ifftshift(x) (the origin moved to the corner first)
        x = torch.fft.ifftshift(real.to(torch.float64))
        if outputs_rfft:
            ft = torch.fft.rfftn(x)
            return torch.fft.fftshift(ft, dim=(0, 1)) if fftshifted else ft
        ft = torch.fft.fftn(x)
        return torch.fft.fftshift(ft) if fftshifted else ft


# ---------------------------------------------------------------------------
# Parameter packing
# ---------------------------------------------------------------------------


def pack_image_params(pose: AbstractPose, image_config: BasicImageConfig,
                      transfer_theory: ContrastTransferTheory | None = None, scale=1.0, n: int | None = None):
    """Build the float64 [n, 32] cjx_image_params records for a batch."""
    q = pose.quaternion()
    ctf = transfer_theory.ctf if transfer_theory is not None else None
    cands = [q if q.ndim > 1 else None, pose.offset_in_angstroms if pose.offset_in_angstroms.ndim > 1 else None,
             image_config.pixel_size, image_config.voltage_in_kilovolts, scale]
    if transfer_theory is not None:
        cands += [ctf.defocus_in_angstroms, ctf.astigmatism_in_angstroms, ctf.astigmatism_angle,
                  ctf.spherical_aberration_in_mm, transfer_theory.amplitude_contrast_ratio,
                  transfer_theory.phase_shift]
        if transfer_theory.envelope is not None:
            cands += list(_envelope_amp_b(transfer_theory.envelope))
    if n is None:
        n = _batch_size(*cands) or 1
    p = nat.empty_params(n)
    R = rot.quat_to_matrix(q)
    p[:, 0:9] = np.broadcast_to(R.reshape(-1, 9) if R.ndim == 3 else R.reshape(1, 9), (n, 9))
    off = pose.offset_in_angstroms
    off = off.reshape(-1, off.shape[-1]) if off.ndim > 1 else off[None]
    off = np.broadcast_to(off, (n, off.shape[-1]))
    p[:, nat.P_SHIFT_X] = off[:, 0]
    p[:, nat.P_SHIFT_Y] = off[:, 1]
    px = _per_image(image_config.pixel_size, n)
    kv = _per_image(image_config.voltage_in_kilovolts, n)
    p[:, nat.P_PIXEL_SIZE] = px
    p[:, nat.P_WAVELENGTH] = C.wavelength_from_kilovolts(kv)
    p[:, nat.P_SCALE] = _per_image(scale, n)
    if transfer_theory is not None:
        df = _per_image(ctf.defocus_in_angstroms, n)
        if off.shape[-1] == 3:
            df = df + off[:, 2]
        p[:, nat.P_DEFOCUS] = df
        p[:, nat.P_ASTIG] = _per_image(ctf.astigmatism_in_angstroms, n)
        p[:, nat.P_ASTIG_ANGLE] = np.deg2rad(_per_image(ctf.astigmatism_angle, n))
        p[:, nat.P_CS] = _per_image(ctf.spherical_aberration_in_mm, n) * 1e7
        ac = _per_image(transfer_theory.amplitude_contrast_ratio, n)
        p[:, nat.P_PHASE_TOTAL] = np.deg2rad(_per_image(transfer_theory.phase_shift, n)) + np.arctan(
            ac / np.sqrt(1.0 - ac**2))
        p[:, nat.P_AC] = ac
        p[:, nat.P_PHASE_SHIFT] = np.deg2rad(_per_image(transfer_theory.phase_shift, n))
        if transfer_theory.envelope is not None:
            amp, b = _envelope_amp_b(transfer_theory.envelope)
            p[:, nat.P_ENV_AMP] = _per_image(amp, n)
            p[:, nat.P_ENV_B] = _per_image(b, n)
    return p


# ---------------------------------------------------------------------------
# Processing order
# ---------------------------------------------------------------------------


def _hilbert_index(x, y, order):
    """Hilbert-curve index of integer points (x, y) in [0, 2^order)^2."""
    x = x.astype(np.int64).copy()
    y = y.astype(np.int64).copy()
    d = np.zeros_like(x)
    s = 1 << (order - 1)
    while s > 0:
        rx = (x & s) > 0
        ry = (y & s) > 0
        d += s * s * ((3 * rx) ^ ry)
        # rotate the quadrant
        swap = ~ry
        flip = swap & rx
        x = np.where(flip, s - 1 - x, x)
        y = np.where(flip, s - 1 - y, y)
        x, y = np.where(swap, y, x), np.where(swap, x, y)
        s >>= 1
    return d


def orientation_order(rotations: np.ndarray, bits: int = 8) -> np.ndarray:
    """Permutation that visits images with similar slice planes together.

    The plane sampled for an image is spanned by R[:, 0] and R[:, 1]; its
    normal R[:, 2] (sign-free: n and -n give the same plane) is mapped to a
    hemisphere, projected with Lambert's equal-area azimuthal projection and
    ordered along a Hilbert curve.  Consecutive images then touch largely the
    same voxels, which the L2 cache serves once.
    """
    R = np.asarray(rotations, np.float64).reshape(-1, 3, 3)
    n = R[:, :, 2].copy()
    flip = (n[:, 2] < 0) | ((n[:, 2] == 0) & (n[:, 1] < 0))
    n[flip] *= -1.0
    k = np.sqrt(2.0 / (1.0 + np.clip(n[:, 2], 0.0, 1.0)))
    px, py = k * n[:, 0], k * n[:, 1]  # disk of radius sqrt(2)
    scale = (1 << bits) - 1
    gx = np.clip(np.round((px / np.sqrt(2.0) + 1.0) * 0.5 * scale), 0, scale)
    gy = np.clip(np.round((py / np.sqrt(2.0) + 1.0) * 0.5 * scale), 0, scale)
    return np.argsort(_hilbert_index(gx, gy, bits), kind="stable").astype(np.int32)


# ---------------------------------------------------------------------------
# Integrator
# ---------------------------------------------------------------------------


class FourierSliceExtraction:
    """Fourier-slice projection of a FourierVoxelGridVolume on the B200.

    cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:26-183
    (trilinear sampling of a FourierVoxelGridVolume, cubic-spline sampling
    of a FourierVoxelSplineVolume; ``correction_mask`` is not implemented).  ``out_of_bounds_mode="fill"`` with ``fill_value`` follows
    the reference; ``"zero_fill_negative"`` fills negative indices too
    (not the reference's rule, see CJX_ZERO_FILL_NEGATIVE).
    """

    is_projection_approximation = True

    def __init__(self, *, outputs_integral: bool = True, correction_mask=None, out_of_bounds_mode: str = "fill",
                 fill_value: complex = 0.0 + 0.0j, use_bricked_layout: bool = True, pair_layout: bool = True):
        if correction_mask is not None:
            raise NotImplementedError("correction_mask is not implemented on the device")
        if out_of_bounds_mode not in ("fill", "zero_fill_negative"):
            raise NotImplementedError(f"out_of_bounds_mode={out_of_bounds_mode!r}")
        self.outputs_integral = outputs_integral
        self.correction_mask = None
        self.out_of_bounds_mode = out_of_bounds_mode
        self.fill_value = complex(fill_value)
        self.use_bricked_layout = use_bricked_layout
        self.pair_layout = pair_layout

    def device_grid(self, volume):
        """(grid tensor, layout flag) the forward and search kernels read.

        Bricked layouts are cached on the volume: the x-pair copy when
        ``pair_layout`` (default), else the plain bricked copy; without
        ``use_bricked_layout`` the reference's C-order array itself.  A
        FourierVoxelSplineVolume gives its coefficients (CJX_GRID_SPLINE) in
        the same three layouts.
        """
        if isinstance(volume, FourierVoxelSplineVolume):
            coef = volume.spline_coefficients
            if not (self.use_bricked_layout and coef.is_cuda):
                return coef, nat.CJX_GRID_SPLINE
            if self.pair_layout:
                return volume.pair_grid(), nat.CJX_GRID_SPLINE | nat.CJX_GRID_BRICKED_PAIRS
            return volume.bricked_grid(), nat.CJX_GRID_SPLINE | nat.CJX_GRID_BRICKED
        grid = volume.fourier_voxel_grid
        if not (self.use_bricked_layout and grid.is_cuda):
            return grid, 0
        if self.pair_layout:
            return volume.pair_grid(), nat.CJX_GRID_BRICKED_PAIRS
        return volume.bricked_grid(), nat.CJX_GRID_BRICKED

    def _base_flags(self):
        return nat.CJX_ZERO_FILL_NEGATIVE if self.out_of_bounds_mode == "zero_fill_negative" else 0

    def _out_columns(self, px, flags):
        return px // 2 + 1

    def run(self, volume: FourierVoxelGridVolume, image_config: BasicImageConfig, params: np.ndarray | None,
            flags: int, *, params_device=None, out=None, workspace=None, stream=None, images_per_chunk=0,
            n=None, order=None, filter=None):
        """Launch the batched kernel; returns a complex64 [n, Py, Px//2+1] CUDA tensor.

        ``params`` (host float64 [n, 32]) is copied to the device unless
        ``params_device`` is given.  ``out`` and ``workspace`` are allocated
        when not supplied.  ``filter`` (an AbstractFilter or array over the
        output grid) is multiplied in inside the kernel's epilogue.
        """
        torch = _torch()
        n_vol = volume.shape[0]
        grid, layout = self.device_grid(volume)
        flags = flags | layout
        if image_config.pad_mode != "constant":
            raise NotImplementedError("only constant padding is implemented on the device")
        py, px = image_config.padded_shape
        desc = nat.make_desc(n_vol, py, px, flags | self._base_flags(), self.fill_value, images_per_chunk)
        if n is None:
            n = params_device.shape[0] if params_device is not None else params.shape[0]
        if params_device is None:
            params_device = torch.as_tensor(params, dtype=torch.float64, device=grid.device)
        if out is None:
            out = torch.empty((n, py, self._out_columns(px, flags)), dtype=torch.complex64, device=grid.device)
        ws_bytes = nat.workspace_size(desc, n)
        if ws_bytes and (workspace is None or workspace.numel() * workspace.element_size() < ws_bytes):
            workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=grid.device)
        if order is not None and not isinstance(order, torch.Tensor):
            order = torch.as_tensor(np.asarray(order, np.int32), device=grid.device)
        fdev = None
        if filter is not None:
            arr = filter.get() if hasattr(filter, "get") else filter
            fdev = torch.as_tensor(np.asarray(arr) if not isinstance(arr, torch.Tensor) else arr,
                                   dtype=torch.float32, device=grid.device).contiguous()
            if tuple(fdev.shape) != tuple(out.shape[-2:]):
                raise ValueError(f"Found that the `filter` was shape {tuple(fdev.shape)}, but expected it to be "
                                 f"shape {tuple(out.shape[-2:])} (the padded Fourier image).")
        nat.slice_ctf_forward(desc, grid, params_device, out, workspace if ws_bytes else None, stream, order,
                              filter=fdev)
        return out

    def integrate(self, volume_representation: FourierVoxelGridVolume, image_config: BasicImageConfig,
                  outputs_real_space: bool = False):
        """cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:78-146."""
        pose = volume_representation.rotation or QuaternionPose()
        scale = image_config.pixel_size if self.outputs_integral else 1.0
        params = pack_image_params(pose, image_config, None, scale=scale)
        out = self.run(volume_representation, image_config, params, 0)
        if pose.batch_size is None and _batch_size(image_config.pixel_size) is None:
            out = out[0]
        if outputs_real_space:
            from . import _postprocess

            return _postprocess.irfftn(out, image_config.padded_shape)
        return out


class EwaldSphereExtraction(FourierSliceExtraction):
    """Ewald-sphere surface extraction on the B200.

    cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:225-516:
    the surface R (q + (lambda / pixel_size) |q|^2 zhat / 2) of a
    FourierVoxelGridVolume (trilinear) or FourierVoxelSplineVolume (cubic
    spline), not reduced to an rfft half plane.  ``integrate`` returns the
    full [Py, Px] spectrum; in an image model with a ContrastTransferTheory
    the contrast follows the reference's non-projection branch
    (cryojax/simulator/_transfer_theory/transfer_theory.py:100-111, 165-255).
    """

    is_projection_approximation = False

    def _base_flags(self):
        return super()._base_flags() | nat.CJX_EWALD_SPHERE

    def _out_columns(self, px, flags):
        return px // 2 + 1 if flags & nat.CJX_APPLY_CTF else px

    def integrate(self, volume_representation, image_config: BasicImageConfig, outputs_real_space: bool = False):
        """cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:269-324."""
        pose = volume_representation.rotation or QuaternionPose()
        scale = image_config.pixel_size if self.outputs_integral else 1.0
        params = pack_image_params(pose, image_config, None, scale=scale)
        out = self.run(volume_representation, image_config, params, 0)
        if pose.batch_size is None and _batch_size(image_config.pixel_size) is None:
            out = out[0]
        if outputs_real_space:
            from . import _postprocess

            # irfftn of the full spectrum reads its first Px//2 + 1 columns
            return _postprocess.irfftn(out[..., : image_config.padded_shape[1] // 2 + 1].contiguous(),
                                       image_config.padded_shape)
        return out


# ---------------------------------------------------------------------------
# Scattering theory and image models
# ---------------------------------------------------------------------------


class WeakPhaseScatteringTheory:
    """cryojax/simulator/_scattering_theory/weak_phase_scattering_theory.py:13-80."""

    def __init__(self, volume_integrator: FourierSliceExtraction, transfer_theory: ContrastTransferTheory,
                 solvent=None):
        if solvent is not None:
            raise NotImplementedError("solvent models are not implemented on the device")
        self.volume_integrator = volume_integrator
        self.transfer_theory = transfer_theory
        self.solvent = None


class AbstractImageModel:
    normalizes_signal: bool = False

    # subclasses set: volume_parametrization, pose, image_config, volume_integrator,
    # transfer_theory (or None), applies_translation, translate_mode, _quantity
    def _scale(self):
        cfg = self.image_config
        s = cfg.pixel_size if self.volume_integrator.outputs_integral else np.float64(1.0)
        if self._quantity:
            s = s * cfg.interaction_constant
        return s

    def _flags(self):
        f = 0
        if self.transfer_theory is not None:
            f |= nat.CJX_APPLY_CTF
            if self.transfer_theory.envelope is not None:
                f |= nat.CJX_APPLY_ENVELOPE
        if self.applies_translation:
            if self.translate_mode != "fft":
                raise ValueError("translate_mode='atom' needs an atom volume, not a FourierVoxelGridVolume")
            f |= nat.CJX_APPLY_TRANSLATION
        if not self.volume_integrator.is_projection_approximation and not (f & nat.CJX_APPLY_CTF):
            raise NotImplementedError("an Ewald-sphere image needs a transfer theory (the integrator alone "
                                      "gives the full spectrum: use EwaldSphereExtraction.integrate)")
        return f

    def image_params(self) -> np.ndarray:
        return pack_image_params(self.pose, self.image_config, self.transfer_theory, scale=self._scale())

    @property
    def batch_size(self):
        return _batch_size(*[None if p is None else p for p in self._batched_fields()])

    def _batched_fields(self):
        tt = self.transfer_theory
        fields = [self.pose.quaternion() if self.pose.quaternion().ndim > 1 else None,
                  self.pose.offset_in_angstroms if self.pose.offset_in_angstroms.ndim > 1 else None,
                  self.image_config.pixel_size, self.image_config.voltage_in_kilovolts]
        if tt is not None:
            fields += [tt.ctf.defocus_in_angstroms, tt.ctf.astigmatism_in_angstroms, tt.ctf.astigmatism_angle,
                       tt.ctf.spherical_aberration_in_mm, tt.amplitude_contrast_ratio, tt.phase_shift]
        return fields

    def get_pose(self):
        return self.pose

    def get_image_config(self):
        return self.image_config

    def compute_fourier_image(self, rng_key=None, *, out=None, workspace=None, stream=None, params_device=None,
                              filter=None):
        """One launch for the whole batch: rotate -> integrate -> CTF -> translate (-> filter).

        cryojax/simulator/_image_model/base_image_model.py:297-328; ``filter``
        is postprocess's Fourier filter, fused into the same launch.
        """
        params = self.image_params()
        img = self.volume_integrator.run(self.volume_parametrization.get_representation(), self.image_config,
                                         params, self._flags(), out=out, workspace=workspace, stream=stream,
                                         params_device=params_device, filter=filter)
        return img if self.batch_size is not None else img[0]

    def simulate(self, rng_key=None, *, removes_padding: bool = True, outputs_real_space: bool = True, mask=None,
                 filter=None):
        """cryojax/simulator/_image_model/base_image_model.py:68-158.

        ``filter`` (over the padded rfft grid) is multiplied into the Fourier
        image inside the device launch; ``mask`` multiplies the real-space
        image after the inverse transform, crop and normalisation.  Without
        ``removes_padding`` neither is applied (as in the reference).
        """
        from . import _postprocess

        cfg = self.image_config
        if not removes_padding:
            fourier_image = self.compute_fourier_image(rng_key)
            return _postprocess.irfftn(fourier_image, cfg.padded_shape) if outputs_real_space else fourier_image
        fourier_image = self.compute_fourier_image(rng_key, filter=filter)
        return _postprocess.postprocess(fourier_image, cfg.shape, cfg.padded_shape,
                                        outputs_real_space=outputs_real_space,
                                        normalizes_signal=self.normalizes_signal, mask=mask)


class LinearImageModel(AbstractImageModel):
    """cryojax/simulator/_image_model/base_image_model.py:216-328."""

    def __init__(self, volume_parametrization, pose, image_config, volume_integrator, transfer_theory, *,
                 applies_translation=True, normalizes_signal=False, signal_region=None, translate_mode="fft"):
        if signal_region is not None:
            raise NotImplementedError("signal_region is not implemented on the device")
        self.volume_parametrization = volume_parametrization
        self.pose = pose
        self.image_config = image_config
        self.volume_integrator = volume_integrator
        self.transfer_theory = transfer_theory
        self.applies_translation = applies_translation
        self.normalizes_signal = normalizes_signal
        self.translate_mode = translate_mode
        self._quantity = False


class ProjectionImageModel(LinearImageModel):
    """cryojax/simulator/_image_model/base_image_model.py:331-432 (no transfer theory)."""

    def __init__(self, volume_parametrization, pose, image_config, volume_integrator, *, applies_translation=True,
                 normalizes_signal=False, signal_region=None, translate_mode="fft"):
        super().__init__(volume_parametrization, pose, image_config, volume_integrator, None,
                         applies_translation=applies_translation, normalizes_signal=normalizes_signal,
                         signal_region=signal_region, translate_mode=translate_mode)


class ContrastImageModel(AbstractImageModel):
    """cryojax/simulator/_image_model/physical_image_model.py:30-137 with WeakPhaseScatteringTheory."""

    def __init__(self, volume_parametrization, pose, image_config, scattering_theory: WeakPhaseScatteringTheory, *,
                 applies_translation=True, normalizes_signal=False, signal_region=None, translate_mode="fft"):
        if signal_region is not None:
            raise NotImplementedError("signal_region is not implemented on the device")
        self.volume_parametrization = volume_parametrization
        self.pose = pose
        self.image_config = image_config
        self.scattering_theory = scattering_theory
        self.volume_integrator = scattering_theory.volume_integrator
        self.transfer_theory = scattering_theory.transfer_theory
        self.applies_translation = applies_translation
        self.normalizes_signal = normalizes_signal
        self.translate_mode = translate_mode
        self._quantity = True


def make_image_model(volume_parametrization, image_config, pose, transfer_theory=None, volume_integrator=None,
                     detector=None, *, applies_translation=True, normalizes_signal=False, signal_region=None,
                     simulates_quantity=False, quantity_mode="contrast", translate_mode="fft"):
    """cryojax/simulator/_api_utils.py:36-223 (Fourier voxel volume routes)."""
    if not isinstance(volume_parametrization, (FourierVoxelGridVolume, FourierVoxelSplineVolume)):
        raise ValueError(
            "Could not select default integrator for volume of type "
            f"{type(volume_parametrization).__name__}: only FourierVoxelGridVolume and FourierVoxelSplineVolume "
            "run on the device")
    if volume_integrator is None:
        volume_integrator = FourierSliceExtraction(outputs_integral=simulates_quantity)
    kw = dict(applies_translation=applies_translation, normalizes_signal=normalizes_signal,
              signal_region=signal_region, translate_mode=translate_mode)
    if transfer_theory is None:
        return ProjectionImageModel(volume_parametrization, pose, image_config, volume_integrator, **kw)
    if simulates_quantity:
        if quantity_mode != "contrast":
            raise NotImplementedError(f"quantity_mode={quantity_mode!r} is not implemented on the device")
        theory = WeakPhaseScatteringTheory(volume_integrator, transfer_theory)
        return ContrastImageModel(volume_parametrization, pose, image_config, theory, **kw)
    return LinearImageModel(volume_parametrization, pose, image_config, volume_integrator, transfer_theory, **kw)
