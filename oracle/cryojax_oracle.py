"""Float64 NumPy restatement of cryoJAX's Fourier-slice + CTF image path.

TEST INFRASTRUCTURE ONLY: the oracle that the CUDA path is checked against.
The product package never imports it.

Every function follows the cryoJAX source file and line range named in its
docstring (paths relative to the cryoJAX project root).  cryoJAX is written
in JAX; JAX is not importable here, so the JAX primitives it calls are
restated with their documented semantics:

* ``jnp.fft.*``  -> ``numpy.fft`` (pocketfft; same conventions, float64).
  For ``irfftn`` of a spectrum whose DC / Nyquist columns are not Hermitian,
  pocketfft (like the ducc FFT behind JAX's CPU backend) transforms the
  leading axes as complex and ignores the imaginary part of the DC and
  Nyquist bins of the last axis.
* ``x.at[idx].get(mode="fill", fill_value=c)`` -> negative indices are first
  wrapped once (``i -> i + n`` for ``-n <= i < 0``, JAX's default
  ``wrap_negative_indices=True``); an index that is still outside
  ``[0, n)`` on any axis yields the fill value.  ``wrap_negative=False``
  gives pure zero fill (selectable for comparison; not the reference).
"""

from __future__ import annotations

import itertools
import math

import numpy as np


# ---------------------------------------------------------------------------
# Physical constants  (cryojax/constants/_physical_constants.py)
# ---------------------------------------------------------------------------

# CODATA values as used through scipy.constants by the reference
_SPEED_OF_LIGHT = 299792458.0
_ELECTRON_MASS = 9.1093837139e-31
_ELEMENTARY_CHARGE = 1.602176634e-19


def wavelength_from_kilovolts(voltage_in_kilovolts):
    """Relativistic electron wavelength in Angstroms.

    cryojax/constants/_physical_constants.py:10-29.
    """
    v = 1000.0 * np.asarray(voltage_in_kilovolts, dtype=np.float64)
    return 12.2639 / (v + 0.97845e-6 * v**2) ** 0.5


def lorentz_factor_from_kilovolts(voltage_in_kilovolts):
    """cryojax/constants/_physical_constants.py:32-49."""
    try:
        import scipy.constants as sc

        c, m0, e = sc.speed_of_light, sc.electron_mass, sc.elementary_charge
    except Exception:  # pragma: no cover - scipy is present in this image
        c, m0, e = _SPEED_OF_LIGHT, _ELECTRON_MASS, _ELEMENTARY_CHARGE
    rest_energy = m0 * c**2
    accelerating_energy = e * (1000.0 * np.asarray(voltage_in_kilovolts, np.float64))
    return 1.0 + accelerating_energy / rest_energy


def interaction_constant_from_kilovolts(voltage_in_kilovolts):
    """sigma_e = lambda * gamma.  cryojax/constants/_physical_constants.py:52-109."""
    return wavelength_from_kilovolts(voltage_in_kilovolts) * lorentz_factor_from_kilovolts(
        voltage_in_kilovolts
    )


# ---------------------------------------------------------------------------
# Coordinate and frequency grids  (cryojax/coordinates/_make_coordinate_grids.py)
# ---------------------------------------------------------------------------


def make_frequency_grid(shape, grid_spacing=1.0, outputs_rfftfreqs=True):
    """2-D frequency grid, zero in the corner; [...,0]=kx, [...,1]=ky.

    cryojax/coordinates/_make_coordinate_grids.py:67-97, 259-298, 301-317.
    """
    if len(shape) != 2:
        raise ValueError("only 2-D frequency grids are restated")
    y = np.fft.fftfreq(shape[0], grid_spacing)
    x = (np.fft.rfftfreq if outputs_rfftfreqs else np.fft.fftfreq)(shape[1], grid_spacing)
    xv, yv = np.meshgrid(x, y, indexing="xy")
    return np.stack([xv, yv], axis=-1)


def make_frequency_slice(shape, grid_spacing=1.0, outputs_rfftfreqs=True):
    """Central kz=0 slice with the zero frequency in the centre; (1, Ny, Nx, 3).

    cryojax/coordinates/_make_coordinate_grids.py:139-198.
    """
    g = make_frequency_grid(shape, grid_spacing, outputs_rfftfreqs=outputs_rfftfreqs)
    g = np.fft.fftshift(g, axes=(0,) if outputs_rfftfreqs else (0, 1))
    g = np.pad(g, ((0, 0), (0, 0), (0, 1)), mode="constant", constant_values=0.0)
    return g[None]


def safe_multiply_by_constant(grid, constant):
    """cryojax/simulator/_image_config.py:406-412."""
    return np.where(grid != 0.0, constant * grid, 0.0)


def padded_frequency_grid_in_angstroms(padded_shape, pixel_size):
    """cryojax/simulator/_image_config.py:177-201 (rfft frequencies / pixel size)."""
    return safe_multiply_by_constant(
        make_frequency_grid(padded_shape, outputs_rfftfreqs=True), 1.0 / pixel_size
    )


def cartesian_to_polar(grid, square=False):
    """theta = atan2(grid[...,0], grid[...,1]).  cryojax/coordinates/_geometry.py:5-32."""
    theta = np.arctan2(grid[..., 0], grid[..., 1])
    k_sqr = np.sum(np.square(grid), axis=-1)
    return (k_sqr, theta) if square else (np.sqrt(k_sqr), theta)


# ---------------------------------------------------------------------------
# Rotations  (cryojax/rotations/_lie_group.py, cryojax/simulator/_pose.py)
# ---------------------------------------------------------------------------


def quat_compose(q0, q1):
    """Hamilton product.  cryojax/rotations/_lie_group.py:103-115."""
    w0, x0, y0, z0 = np.moveaxis(np.asarray(q0, np.float64), -1, 0)
    w1, x1, y1, z1 = np.moveaxis(np.asarray(q1, np.float64), -1, 0)
    return np.stack(
        [
            -x0 * x1 - y0 * y1 - z0 * z1 + w0 * w1,
            x0 * w1 + y0 * z1 - z0 * y1 + w0 * x1,
            -x0 * z1 + y0 * w1 + z0 * x1 + w0 * y1,
            x0 * y1 - y0 * x1 + z0 * w1 + w0 * z1,
        ],
        axis=-1,
    )


def quat_inverse(q):
    """cryojax/rotations/_lie_group.py:117-119."""
    return np.asarray(q, np.float64) * np.array([1.0, -1.0, -1.0, -1.0])


def quat_normalize(q):
    """cryojax/rotations/_lie_group.py:316-318."""
    q = np.asarray(q, np.float64)
    return q / np.linalg.norm(q, axis=-1, keepdims=True)


def quat_apply(q, v):
    """q (x) (0, v) (x) q^-1, vectorised over the leading axes of v.

    cryojax/rotations/_lie_group.py:97-101.
    """
    v = np.asarray(v, np.float64)
    padded = np.concatenate([np.zeros(v.shape[:-1] + (1,)), v], axis=-1)
    q = np.broadcast_to(np.asarray(q, np.float64), padded.shape)
    return quat_compose(quat_compose(q, padded), quat_inverse(q))[..., 1:]


def quat_as_matrix(q):
    """cryojax/rotations/_lie_group.py:221-232."""
    q = np.asarray(q, np.float64)
    norm = q @ q
    q = q * np.sqrt(2.0 / norm)
    q = np.outer(q, q)
    return np.array(
        [
            [1.0 - q[2, 2] - q[3, 3], q[1, 2] - q[3, 0], q[1, 3] + q[2, 0]],
            [q[1, 2] + q[3, 0], 1.0 - q[1, 1] - q[3, 3], q[2, 3] - q[1, 0]],
            [q[1, 3] - q[2, 0], q[2, 3] + q[1, 0], 1.0 - q[1, 1] - q[2, 2]],
        ]
    )


def so3_exp(tangent):
    """Exponential map to a quaternion.  cryojax/rotations/_lie_group.py:234-271."""
    tangent = np.asarray(tangent, np.float64)
    theta_squared = tangent @ tangent
    theta_pow_4 = theta_squared * theta_squared
    use_taylor = theta_squared < 1e-10
    safe_theta = np.sqrt(1.0 if use_taylor else theta_squared)
    safe_half_theta = 0.5 * safe_theta
    if use_taylor:
        real = 1.0 - theta_squared / 8.0 + theta_pow_4 / 384.0
        imag = 0.5 - theta_squared / 48.0 + theta_pow_4 / 3840.0
    else:
        real = np.cos(safe_half_theta)
        imag = np.sin(safe_half_theta) / safe_theta
    return np.concatenate([[real], imag * tangent])


def euler_pose_quaternion(phi_angle, theta_angle, psi_angle):
    """zyz extrinsic, degrees: R3 @ R2 @ R1.  cryojax/simulator/_pose.py:257-272."""
    phi, theta, psi = np.deg2rad([phi_angle, theta_angle, psi_angle])
    r1 = so3_exp(np.array([0.0, 0.0, phi]))
    r2 = so3_exp(np.array([0.0, theta, 0.0]))
    r3 = so3_exp(np.array([0.0, 0.0, psi]))
    return quat_compose(quat_compose(r3, r2), r1)


def axis_angle_pose_quaternion(euler_vector_in_degrees):
    """cryojax/simulator/_pose.py:387-398."""
    return so3_exp(np.deg2rad(np.asarray(euler_vector_in_degrees, np.float64)))


def quaternion_pose_rotation(wxyz):
    """QuaternionPose.rotation = SO3(wxyz).normalize().  cryojax/simulator/_pose.py:324-330."""
    return quat_normalize(wxyz)


def sample_uniform_quaternion(u1, u2, u3):
    """Shoemake's uniform S^3 sample from u1~U(0,1), u2,u3~U(0,2pi).

    cryojax/rotations/_lie_group.py:320-341 (same formula; the uniforms are
    drawn by the caller).
    """
    a = np.sqrt(1.0 - u1)
    b = np.sqrt(u1)
    return np.stack([a * np.sin(u2), a * np.cos(u2), b * np.sin(u3), b * np.cos(u3)], -1)


# ---------------------------------------------------------------------------
# FFT conventions and edges  (cryojax/ndimage/_fft.py, _edges.py)
# ---------------------------------------------------------------------------


def fftn(x, s=None, axes=None):
    """cryojax/ndimage/_fft.py:34-55."""
    axes = _axes_for(x, s, axes)
    return np.fft.fftn(np.fft.ifftshift(x, axes=axes), s=s, axes=axes)


def ifftn(ft, s=None, axes=None):
    """cryojax/ndimage/_fft.py:11-31."""
    axes = _axes_for(ft, s, axes)
    return np.fft.fftshift(np.fft.ifftn(ft, s=s, axes=axes), axes=axes)


def _axes_for(x, s, axes):
    if axes is None and s is not None:
        return tuple(range(np.ndim(x) - len(s), np.ndim(x)))
    return axes


def rfftn(x, s=None, axes=None):
    """cryojax/ndimage/_fft.py:80-99."""
    axes = _axes_for(x, s, axes)
    return np.fft.rfftn(np.fft.ifftshift(x, axes=axes), s=s, axes=axes)


def irfftn(ft, s=None, axes=None):
    """cryojax/ndimage/_fft.py:57-77."""
    axes = _axes_for(ft, s, axes)
    return np.fft.fftshift(np.fft.irfftn(ft, s=s, axes=axes), axes=axes)


def get_left_vs_right_pad(pad_dim, image_dim):
    """cryojax/ndimage/_edges.py:175-185."""
    pad = pad_dim - image_dim
    if pad_dim % 2 == 0 and image_dim % 2 == 0:
        return pad // 2, pad // 2
    if pad_dim % 2 == 1 and image_dim % 2 == 0:
        return pad // 2, pad // 2 + 1
    if pad_dim % 2 == 0 and image_dim % 2 == 1:
        return pad // 2 + 1, pad // 2
    return pad // 2, pad // 2


def pad_to_shape(x, shape, mode="constant"):
    """cryojax/ndimage/_edges.py:110-147."""
    padding = tuple(get_left_vs_right_pad(s, d) for s, d in zip(shape, x.shape))
    return np.pad(x, padding, mode=mode)


def crop_to_shape(x, shape):
    """Centre crop.  cryojax/ndimage/_edges.py:15-62."""
    slices = []
    for n, h in zip(x.shape, shape):
        c = n // 2
        slices.append(slice(c - h // 2, c + h // 2 + h % 2))
    return x[tuple(slices)]


def resize_with_crop_or_pad(image, shape, mode="constant"):
    """cryojax/ndimage/_edges.py:150-172."""
    n1, n2 = image.shape
    m1, m2 = shape
    if n1 >= m1 and n2 >= m2:
        return crop_to_shape(image, shape)
    if n1 <= m1 and n2 <= m2:
        return pad_to_shape(image, shape, mode=mode)
    if n1 <= m1 and n2 >= m2:
        return pad_to_shape(crop_to_shape(image, (n1, m2)), (m1, m2), mode=mode)
    return pad_to_shape(crop_to_shape(image, (m1, n2)), (m1, m2), mode=mode)


# ---------------------------------------------------------------------------
# rfft half-plane utilities  (cryojax/ndimage/_fourier_utils.py)
# ---------------------------------------------------------------------------


def enforce_self_conjugate_rfftn_components(
    rfftn_array, shape, includes_zero_frequency=False, mode="zero"
):
    """2-D branch.  cryojax/ndimage/_fourier_utils.py:60-132."""
    if mode == "zero":
        fn = lambda a: 0.0  # noqa: E731
    elif mode == "one":
        fn = lambda a: 1.0  # noqa: E731
    elif mode == "real":
        fn = lambda a: a.real  # noqa: E731
    else:
        raise NotImplementedError(mode)
    out = np.array(rfftn_array, copy=True)
    y_dim, x_dim = shape
    if includes_zero_frequency:
        out[0, 0] = fn(out[0, 0])
    if y_dim % 2 == 0:
        out[y_dim // 2, 0] = fn(out[y_dim // 2, 0])
    if x_dim % 2 == 0:
        out[0, x_dim // 2] = fn(out[0, x_dim // 2])
    if y_dim % 2 == 0 and x_dim % 2 == 0:
        out[y_dim // 2, x_dim // 2] = fn(out[y_dim // 2, x_dim // 2])
    return out


def convert_fftn_to_rfftn(fftn_array, mode="zero"):
    """cryojax/ndimage/_fourier_utils.py:6-57."""
    shape = fftn_array.shape
    out = fftn_array[:, : shape[-1] // 2 + 1]
    if mode is not None:
        out = enforce_self_conjugate_rfftn_components(out, shape, False, mode)
    return out


# ---------------------------------------------------------------------------
# Interpolation  (cryojax/ndimage/_map_coordinates.py)
# ---------------------------------------------------------------------------


def map_coordinates_linear(grid, coordinates, cval=0.0, wrap_negative=True):
    """order=1, mode="fill" trilinear sampling.

    cryojax/ndimage/_map_coordinates.py:85-123 (corner loop) and 168-175
    (lower = floor(c), w_hi = c - lower, w_lo = 1 - w_hi).  Each corner is
    fetched with ``grid.at[idx].get(mode="fill", fill_value=cval)``
    (:117): indices in [-n, 0) wrap once, anything else outside [0, n)
    yields ``cval``.
    """
    nodes = []
    for c in coordinates:
        c = np.asarray(c, np.float64)
        lower = np.floor(c)
        w_hi = c - lower
        w_lo = 1.0 - w_hi
        idx = lower.astype(np.int64)
        nodes.append([(idx, w_lo), (idx + 1, w_hi)])
    out = 0.0
    for items in itertools.product(*nodes):
        valid = True
        norm_idx = []
        weight = 1.0
        for axis, (idx, w) in enumerate(items):
            n = grid.shape[axis]
            if wrap_negative:
                i = np.where(idx < 0, idx + n, idx)
            else:
                i = idx
            valid = valid & (i >= 0) & (i < n)
            norm_idx.append(np.clip(i, 0, n - 1))
            weight = weight * w
        contribution = np.where(valid, grid[tuple(norm_idx)], cval)
        out = out + weight * contribution
    return np.asarray(out).astype(grid.dtype)


def compute_spline_coefficients(data):
    """Cubic B-spline coefficients, one tridiagonal solve per axis line.

    cryojax/ndimage/_map_coordinates.py:71-82, 179-215: along each axis
    (last axis first) a line d of length n gets c2 = d[0] / 6,
    c_{n+2} = d[-1] / 6, the interior cs from tridiag(1, 4, 1) cs = d[1:-1]
    with d[1] -= c2 and d[-2] -= c_{n+2} (a banded solve here, lineax's
    TridiagonalLinearOperator there), then c1 = 2 c2 - cs[0] and
    c_{n+3} = 2 c_{n+2} - cs[-1]: n + 2 coefficients per line.
    """
    from scipy.linalg import solve_banded

    out = np.asarray(data, np.complex128)
    for axis in reversed(range(out.ndim)):
        x = np.moveaxis(out, axis, 0)
        n = x.shape[0]
        rest = x.shape[1:]
        x = x.reshape(n, -1)
        c2, cnp2 = x[0] / 6.0, x[-1] / 6.0
        y = x[1:-1].copy()
        y[0] -= c2
        y[-1] -= cnp2
        m = n - 2
        ab = np.zeros((3, m))
        ab[0, 1:] = 1.0
        ab[1, :] = 4.0
        ab[2, :-1] = 1.0
        cs = solve_banded((1, 1), ab, y)
        res = np.concatenate([(2 * c2 - cs[0])[None], c2[None], cs, cnp2[None], (2 * cnp2 - cs[-1])[None]], 0)
        out = np.moveaxis(res.reshape((n + 2,) + rest), 0, axis)
    return out


def spline_basis(t):
    """cryojax/ndimage/_map_coordinates.py:217-225 (unnormalised cubic B-spline: 4 at 0, 1 at +-1)."""
    at = np.abs(t)
    return np.where(at >= 1, np.where(at <= 2, (2 - at) ** 3, 0.0), 4 - 6 * at**2 + 3 * at**3)


def map_coordinates_spline(coefficients, coordinates, cval=0.0, wrap_negative=True):
    """Cubic-spline sampling, mode="fill".

    cryojax/ndimage/_map_coordinates.py:48-68, 126-142, 228-250: for a
    coordinate c the taps are the coefficient indices floor(c) + {0, 1, 2, 3}
    along each axis with weights spline_basis(c - i + 1); each tap is read
    with ``.at[idx].get(mode="fill", fill_value=cval)`` (an index in [-n, 0)
    wraps once, anything else outside [0, n) reads cval).
    """
    axes = []
    for c in coordinates:
        c = np.asarray(c, np.float64)
        f = np.floor(c).astype(np.int64)
        axes.append([(f + t, spline_basis(c - (f + t) + 1)) for t in range(4)])
    out = 0.0
    for items in itertools.product(*axes):
        valid = True
        idx = []
        weight = 1.0
        for axis, (i, w) in enumerate(items):
            n = coefficients.shape[axis]
            j = np.where(i < 0, i + n, i) if wrap_negative else i
            valid = valid & (j >= 0) & (j < n)
            idx.append(np.clip(j, 0, n - 1))
            weight = weight * w
        out = out + weight * np.where(valid, coefficients[tuple(idx)], cval)
    return np.asarray(out).astype(np.complex128)


# ---------------------------------------------------------------------------
# Volume and Fourier-slice extraction
# (cryojax/simulator/_volume/representations/voxel_volume.py,
#  cryojax/simulator/_volume_integrator/fourier_voxel_extract.py)
# ---------------------------------------------------------------------------


def fourier_voxel_grid_from_real_voxel_grid(real_voxel_grid, pad_scale=1.0, pad_mode="constant"):
    """Returns (centred full FFT grid, frequency slice in pixels).

    cryojax/simulator/_volume/representations/voxel_volume.py:69-119.
    """
    real = np.asarray(real_voxel_grid, np.float64)
    if pad_scale < 1.0:
        raise ValueError("`pad_scale` must be greater than 1.0")
    padded_shape = tuple(int(s * pad_scale) for s in real.shape)
    padded = pad_to_shape(real, padded_shape, mode=pad_mode)
    grid = np.fft.fftshift(fftn(padded))
    frequency_slice = make_frequency_slice(padded_shape[:-1], outputs_rfftfreqs=False)
    return grid, frequency_slice


def rotate_frequency_slice(frequency_slice, wxyz):
    """AbstractPose.rotate_coordinates(inverse=False) with a unit quaternion.

    cryojax/simulator/_volume/representations/voxel_volume.py:31-37,
    cryojax/simulator/_pose.py:29-66.
    """
    return quat_apply(wxyz, frequency_slice)


def extract_surface_from_voxel_grid(grid, frequency_coordinates, cval=0.0, wrap_negative=True, spline=False):
    """cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:519-544.

    With ``spline`` the grid holds cubic-spline coefficients ((N+2)^3) and
    the surface is sampled with map_coordinates_spline (:531-534).
    """
    n = frequency_coordinates.shape[1]
    logical = frequency_coordinates * n + n // 2
    k_z, k_y, k_x = np.moveaxis(logical, -1, 0)
    if spline:
        surface = map_coordinates_spline(grid, (k_x, k_y, k_z), cval, wrap_negative)[0]
    else:
        surface = map_coordinates_linear(grid, (k_x, k_y, k_z), cval, wrap_negative)[0]
    return np.fft.ifftshift(surface)


def extract_slice(grid, frequency_coordinates, cval=0.0, wrap_negative=True, spline=False):
    """cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:428-457 (grid and spline)."""
    return convert_fftn_to_rfftn(
        extract_surface_from_voxel_grid(grid, frequency_coordinates, cval, wrap_negative, spline),
        mode="real",
    )


def fourier_slice_integrate(
    grid,
    rotated_frequency_slice,
    padded_shape,
    pixel_size,
    *,
    outputs_integral=True,
    pad_mode="constant",
    cval=0.0,
    outputs_real_space=False,
    wrap_negative=True,
    spline=False,
):
    """FourierSliceExtraction.integrate for a FourierVoxelGridVolume
    (or, with ``spline``, a FourierVoxelSplineVolume's coefficients).

    cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:78-146.
    """
    n = rotated_frequency_slice.shape[1]
    m = n + 2 if spline else n
    if grid.shape != (m, m, m):
        raise AttributeError("Only cubic boxes are supported for fourier slice extraction.")
    proj = extract_slice(grid, rotated_frequency_slice, cval, wrap_negative, spline)
    if tuple(padded_shape) != (n, n):
        proj = rfftn(resize_with_crop_or_pad(irfftn(proj, s=(n, n)), tuple(padded_shape), pad_mode))
    if outputs_integral:
        proj = proj * pixel_size
    return irfftn(proj, s=tuple(padded_shape)) if outputs_real_space else proj


def ewald_sphere_frequencies(rotated_frequency_slice, voxel_size, wavelength):
    """Ewald-sphere surface through a rotated frequency slice (cycles/pixel).

    cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:489-516:
    zhat = xhat x yhat from the slice's own (unit-normalised) in-plane axes,
    q_surface = q + (wavelength / voxel_size) |q|^2 zhat / 2.
    """
    corner = np.fft.ifftshift(rotated_frequency_slice, axes=(0, 1, 2))
    xhat, yhat = corner[0, 0, 1, :], corner[0, 1, 0, :]
    xhat = xhat / np.linalg.norm(xhat)
    yhat = yhat / np.linalg.norm(yhat)
    zhat = np.cross(xhat, yhat)
    q_squared = np.sum(rotated_frequency_slice**2, axis=-1)
    return rotated_frequency_slice + (wavelength / voxel_size) * (q_squared[..., None] * zhat) / 2


def ewald_integrate(
    grid,
    rotated_frequency_slice,
    padded_shape,
    pixel_size,
    wavelength,
    *,
    outputs_integral=True,
    pad_mode="constant",
    cval=0.0,
    wrap_negative=True,
    spline=False,
):
    """EwaldSphereExtraction.integrate: the full (not rfft) complex surface.

    cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:269-324,
    455-486: sample the curved surface (trilinear, or cubic spline from
    coefficients), then for padded_shape != (N, N)
    fftn(crop_or_pad(ifftn(surface))) and the pixel-size factor.
    """
    n = rotated_frequency_slice.shape[1]
    m = n + 2 if spline else n
    if grid.shape != (m, m, m):
        raise AttributeError("Only cubic boxes are supported for fourier slice extraction.")
    freqs = ewald_sphere_frequencies(rotated_frequency_slice, pixel_size, wavelength)
    surface = extract_surface_from_voxel_grid(grid, freqs, cval, wrap_negative, spline)
    if tuple(padded_shape) != (n, n):
        surface = fftn(resize_with_crop_or_pad(ifftn(surface, s=(n, n)), tuple(padded_shape), pad_mode))
    if outputs_integral:
        surface = surface * pixel_size
    return surface


def _ewald_propagate(pos, neg, ac, sin, cos):
    """cryojax/simulator/_transfer_theory/transfer_theory.py:245-255."""
    w1, w2 = ac, np.sqrt(1.0 - ac**2)
    sr, si = pos.real + neg.real, pos.imag + neg.imag
    dr, di = neg.real - pos.real, pos.imag - neg.imag
    return 0.5 * ((w2 * sr + w1 * si) * sin + (w2 * si - w1 * sr) * cos
                  + 1.0j * ((w2 * di + w1 * dr) * sin + (w2 * dr - w1 * di) * cos))


def compute_contrast_from_ewald_sphere(object_spectrum, phase_shifts, amplitude_contrast_ratio, padded_shape):
    """Contrast (rfft half plane) from a full Ewald-sphere object spectrum.

    cryojax/simulator/_transfer_theory/transfer_theory.py:165-242: every
    half-plane frequency pairs the spectrum at +q with the spectrum at -q;
    the even-size Nyquist column uses conj(O[-y, Nyq]) as its +q partner,
    the x = 0 column is filled from its y > 0 half by Hermitian symmetry
    (its even-size Nyquist row likewise from conj(O[Ny, 0])).
    ``phase_shifts`` are chi(q) - deg2rad(phase_shift) on the rfft grid.
    """
    ny, nx = padded_shape
    ac = float(amplitude_contrast_ratio)
    sin, cos = np.sin(phase_shifts), np.cos(phase_shifts)
    hx, hy = nx // 2 + nx % 2, ny // 2 + ny % 2  # first negative-frequency index
    out = np.empty((ny, nx // 2 + 1), np.complex128)
    # y >= 1, x >= 1
    pos = object_spectrum[1:, 1:hx]
    neg = object_spectrum[1:, hx:][::-1, ::-1]
    if nx % 2 == 0:
        pos = np.concatenate([pos, np.conj(neg[:, -1:])], axis=1)
    out[1:, 1:] = _ewald_propagate(pos, neg, ac, sin[1:, 1:], cos[1:, 1:])
    # y = 0, x >= 1
    pos0 = object_spectrum[0, 1:hx]
    neg0 = object_spectrum[0, hx:][::-1]
    if nx % 2 == 0:
        pos0 = np.concatenate([pos0, np.conj(neg0[-1:])])
    out[0, 1:] = _ewald_propagate(pos0, neg0, ac, sin[0, 1:nx // 2 + 1], cos[0, 1:nx // 2 + 1])
    # x = 0
    posy = object_spectrum[1:hy, 0]
    negy = object_spectrum[hy:, 0][::-1]
    if ny % 2 == 0:
        posy = np.concatenate([posy, np.conj(negy[-1:])])
    cy = _ewald_propagate(posy, negy, ac, sin[1:ny // 2 + 1, 0], cos[1:ny // 2 + 1, 0])
    c00 = _ewald_propagate(object_spectrum[0, 0], object_spectrum[0, 0], ac, sin[0, 0], cos[0, 0])
    out[:, 0] = np.concatenate([[c00], cy if ny % 2 == 1 else cy[:-1], np.conj(cy[::-1])])
    return out


def make_1d_coordinate_grid(size, grid_spacing=1.0):
    """(i - size//2) * spacing.  cryojax/coordinates/_make_coordinate_grids.py:201-223, 301-317."""
    return np.fft.fftshift(np.fft.fftfreq(size, 1.0 / grid_spacing)) * size


def render_gaussian_mixture(shape, voxel_size, positions, amplitudes, variances):
    """Voxel-averaged Gaussian mixture on a real-space grid (z, y, x).

    cryojax/simulator/_volume_rendering/gaussian_rendering.py:196-336:
    B = 8 pi^2 variance, s = 2 pi / sqrt(B); per axis the integral of each
    Gaussian over voxel i is erf(s (L_i - p + dx)) - erf(s (L_i - p)) with
    L_i = c_i - dx / 2 the voxel's left edge; the voxel value is
    sum over atoms and Gaussians of a / (2 dx)^3 times the three axis
    integrals.  Evaluated densely (every voxel, every Gaussian) in float64.
    """
    from scipy.special import erf

    positions = np.asarray(positions, np.float64).reshape(-1, 3)
    amplitudes = np.asarray(amplitudes, np.float64).reshape(positions.shape[0], -1)
    variances = np.broadcast_to(np.asarray(variances, np.float64).reshape(positions.shape[0], -1), amplitudes.shape)
    b_factors = 8.0 * np.pi**2 * variances
    scaling = 2.0 * np.pi / np.sqrt(b_factors)  # (n, g)
    nz, ny, nx = shape
    integrals = []
    for axis, size in ((0, nx), (1, ny), (2, nz)):
        left = make_1d_coordinate_grid(size, voxel_size) - voxel_size / 2
        delta = left[:, None] - positions[None, :, axis]  # (size, n)
        integrals.append(erf(scaling[None] * (delta + voxel_size)[:, :, None])
                         - erf(scaling[None] * delta[:, :, None]))  # (size, n, g)
    gx, gy, gz = integrals
    prefactor = amplitudes / (2.0 * voxel_size) ** 3
    return np.einsum("xng,yng,zng,ng->zyx", gx, gy, gz, prefactor, optimize=True)


# ---------------------------------------------------------------------------
# CTF and transfer theory  (cryojax/simulator/_transfer_theory/)
# ---------------------------------------------------------------------------


def compute_phase_shifts_with_spherical_aberration(
    frequency_grid_in_angstroms,
    defocus_in_angstroms,
    astigmatism_in_angstroms,
    astigmatism_angle_rad,
    wavelength_in_angstroms,
    spherical_aberration_in_angstroms,
):
    """chi(q).  cryojax/simulator/_transfer_theory/common_functions.py:9-30."""
    k_sqr, azimuth = cartesian_to_polar(frequency_grid_in_angstroms, square=True)
    defocus = defocus_in_angstroms + 0.5 * astigmatism_in_angstroms * np.cos(
        2.0 * (azimuth - astigmatism_angle_rad)
    )
    defocus_phase_shifts = -0.5 * defocus * wavelength_in_angstroms * k_sqr
    aberration_phase_shifts = (
        0.25 * spherical_aberration_in_angstroms * (wavelength_in_angstroms**3) * (k_sqr**2)
    )
    return (2 * np.pi) * (defocus_phase_shifts + aberration_phase_shifts)


def amplitude_contrast_phase_shift(amplitude_contrast_ratio):
    """cryojax/simulator/_transfer_theory/common_functions.py:34-40."""
    ac = float(amplitude_contrast_ratio)
    return np.arctan(ac / np.sqrt(1.0 - ac**2))


def astigmatic_ctf(
    frequency_grid_in_angstroms,
    voltage_in_kilovolts,
    *,
    defocus_in_angstroms=10000.0,
    astigmatism_in_angstroms=0.0,
    astigmatism_angle=0.0,
    spherical_aberration_in_mm=2.7,
    amplitude_contrast_ratio=0.1,
    phase_shift=0.0,
    defocus_offset=None,
):
    """AbstractCTF.__call__(outputs_exp=False) for AstigmaticCTF.

    cryojax/simulator/_transfer_theory/transfer_function.py:27-82, 130-169.
    """
    wavelength = wavelength_from_kilovolts(voltage_in_kilovolts)
    defocus = defocus_in_angstroms if defocus_offset is None else defocus_in_angstroms + defocus_offset
    chi = compute_phase_shifts_with_spherical_aberration(
        frequency_grid_in_angstroms,
        defocus,
        astigmatism_in_angstroms,
        np.deg2rad(astigmatism_angle),
        wavelength,
        spherical_aberration_in_mm * 1e7,
    )
    return np.sin(chi - (np.deg2rad(phase_shift) + amplitude_contrast_phase_shift(amplitude_contrast_ratio)))


def fourier_gaussian_envelope(frequency_grid, amplitude=1.0, b_factor=1.0):
    """FourierGaussian envelope.  cryojax/ndimage/operators/_fourier_operator.py:183-234."""
    k_sqr = np.sum(frequency_grid**2, axis=-1)
    return amplitude * np.exp(-0.25 * b_factor * k_sqr)


# ---------------------------------------------------------------------------
# Translation  (cryojax/simulator/_pose.py:68-114)
# ---------------------------------------------------------------------------


def translation_operator(frequency_grid_in_angstroms, offset_xy):
    """exp(-2 pi i (qx tx + qy ty)).  cryojax/simulator/_pose.py:97-114."""
    xy = np.asarray(offset_xy, np.float64)[0:2]
    return np.exp(-1.0j * (2 * np.pi * np.matmul(frequency_grid_in_angstroms, xy)))


def translate_image(fourier_image, operator, shape):
    """cryojax/simulator/_pose.py:68-95."""
    fourier_image = enforce_self_conjugate_rfftn_components(fourier_image, shape, False, "zero")
    return fourier_image * operator


# ---------------------------------------------------------------------------
# Image model  (cryojax/simulator/_image_model/base_image_model.py)
# ---------------------------------------------------------------------------


class ImageSpec:
    """Plain container for one image's parameters (pose, CTF, config)."""

    def __init__(
        self,
        *,
        shape,
        pixel_size,
        voltage_in_kilovolts=300.0,
        padded_shape=None,
        pad_mode="constant",
        wxyz=(1.0, 0.0, 0.0, 0.0),
        offset_in_angstroms=(0.0, 0.0),
        defocus_in_angstroms=10000.0,
        astigmatism_in_angstroms=0.0,
        astigmatism_angle=0.0,
        spherical_aberration_in_mm=2.7,
        amplitude_contrast_ratio=0.1,
        phase_shift=0.0,
        envelope_b_factor=None,
        envelope_amplitude=1.0,
    ):
        self.shape = tuple(shape)
        self.padded_shape = tuple(padded_shape) if padded_shape is not None else tuple(shape)
        self.pixel_size = float(pixel_size)
        self.voltage_in_kilovolts = float(voltage_in_kilovolts)
        self.pad_mode = pad_mode
        self.wxyz = np.asarray(wxyz, np.float64)
        self.offset_in_angstroms = np.asarray(offset_in_angstroms, np.float64)
        self.defocus_in_angstroms = float(defocus_in_angstroms)
        self.astigmatism_in_angstroms = float(astigmatism_in_angstroms)
        self.astigmatism_angle = float(astigmatism_angle)
        self.spherical_aberration_in_mm = float(spherical_aberration_in_mm)
        self.amplitude_contrast_ratio = float(amplitude_contrast_ratio)
        self.phase_shift = float(phase_shift)
        self.envelope_b_factor = envelope_b_factor
        self.envelope_amplitude = envelope_amplitude


def compute_fourier_image(
    grid,
    frequency_slice,
    spec: ImageSpec,
    *,
    outputs_integral=False,
    simulates_quantity=False,
    applies_translation=True,
    apply_ctf=True,
    cval=0.0,
    wrap_negative=True,
    spline=False,
    ewald=False,
):
    """LinearImageModel / ContrastImageModel.compute_fourier_image.

    cryojax/simulator/_image_model/base_image_model.py:297-328 (linear) and
    cryojax/simulator/_image_model/physical_image_model.py:108-137 with
    cryojax/simulator/_scattering_theory/weak_phase_scattering_theory.py:37-80
    (contrast: integral times the interaction constant).  ``apply_ctf=False``
    is ProjectionImageModel (:412-432).  Order: rotate -> integrate -> CTF ->
    translate.  ``ewald``: EwaldSphereExtraction as the integrator and
    ContrastTransferTheory's non-projection branch
    (cryojax/simulator/_transfer_theory/transfer_theory.py:100-111); without
    the CTF it returns EwaldSphereExtraction.integrate's full spectrum.
    """
    rotated = rotate_frequency_slice(frequency_slice, quaternion_pose_rotation(spec.wxyz))
    if ewald:
        return _compute_fourier_image_ewald(grid, rotated, spec, outputs_integral, simulates_quantity,
                                            applies_translation, apply_ctf, cval, wrap_negative, spline)
    proj = fourier_slice_integrate(
        grid,
        rotated,
        spec.padded_shape,
        spec.pixel_size,
        outputs_integral=outputs_integral,
        pad_mode=spec.pad_mode,
        cval=cval,
        wrap_negative=wrap_negative,
        spline=spline,
    )
    if simulates_quantity:
        proj = interaction_constant_from_kilovolts(spec.voltage_in_kilovolts) * proj
    freqs = padded_frequency_grid_in_angstroms(spec.padded_shape, spec.pixel_size)
    if apply_ctf:
        offset_z = spec.offset_in_angstroms[2] if spec.offset_in_angstroms.shape[0] == 3 else None
        ctf = astigmatic_ctf(
            freqs,
            spec.voltage_in_kilovolts,
            defocus_in_angstroms=spec.defocus_in_angstroms,
            astigmatism_in_angstroms=spec.astigmatism_in_angstroms,
            astigmatism_angle=spec.astigmatism_angle,
            spherical_aberration_in_mm=spec.spherical_aberration_in_mm,
            amplitude_contrast_ratio=spec.amplitude_contrast_ratio,
            phase_shift=spec.phase_shift,
            defocus_offset=offset_z,
        )
        proj = ctf * proj
        if spec.envelope_b_factor is not None:
            proj = proj * fourier_gaussian_envelope(freqs, spec.envelope_amplitude, spec.envelope_b_factor)
    if applies_translation:
        proj = translate_image(proj, translation_operator(freqs, spec.offset_in_angstroms), spec.padded_shape)
    return proj


def _compute_fourier_image_ewald(grid, rotated, spec, outputs_integral, simulates_quantity, applies_translation,
                                 apply_ctf, cval, wrap_negative, spline):
    wavelength = wavelength_from_kilovolts(spec.voltage_in_kilovolts)
    obj = ewald_integrate(grid, rotated, spec.padded_shape, spec.pixel_size, wavelength,
                          outputs_integral=outputs_integral, pad_mode=spec.pad_mode, cval=cval,
                          wrap_negative=wrap_negative, spline=spline)
    if simulates_quantity:
        obj = interaction_constant_from_kilovolts(spec.voltage_in_kilovolts) * obj
    if not apply_ctf:
        if applies_translation:
            raise NotImplementedError("the Ewald spectrum is a full plane; translation applies to the contrast")
        return obj
    freqs = padded_frequency_grid_in_angstroms(spec.padded_shape, spec.pixel_size)
    offset_z = spec.offset_in_angstroms[2] if spec.offset_in_angstroms.shape[0] == 3 else None
    defocus = spec.defocus_in_angstroms if offset_z is None else spec.defocus_in_angstroms + offset_z
    chi = compute_phase_shifts_with_spherical_aberration(
        freqs, defocus, spec.astigmatism_in_angstroms, np.deg2rad(spec.astigmatism_angle), wavelength,
        spec.spherical_aberration_in_mm * 1e7) - np.deg2rad(spec.phase_shift)
    img = compute_contrast_from_ewald_sphere(obj, chi, spec.amplitude_contrast_ratio, spec.padded_shape)
    if spec.envelope_b_factor is not None:
        img = img * fourier_gaussian_envelope(freqs, spec.envelope_amplitude, spec.envelope_b_factor)
    if applies_translation:
        img = translate_image(img, translation_operator(freqs, spec.offset_in_angstroms), spec.padded_shape)
    return img


def postprocess(fourier_image, spec: ImageSpec, *, outputs_real_space=True, normalizes_signal=False, mask=None,
                filter=None):
    """AbstractImageModel.postprocess with optional mask and filter arrays.

    cryojax/simulator/_image_model/base_image_model.py:107-158, 184-192:
    filter (times the padded Fourier image) -> irfftn -> crop -> normalise
    -> mask (times the real-space image).
    """
    if filter is not None:
        fourier_image = fourier_image * filter
    if mask is None and spec.padded_shape == spec.shape and not normalizes_signal:
        return irfftn(fourier_image, s=spec.shape) if outputs_real_space else fourier_image
    image = irfftn(fourier_image, s=spec.padded_shape)
    if spec.padded_shape != spec.shape:
        image = crop_to_shape(image, spec.shape)
    if normalizes_signal:
        image = (image - image.mean()) / image.std()
    if mask is not None:
        image = image * mask
    return image if outputs_real_space else rfftn(image)


def simulate(grid, frequency_slice, spec: ImageSpec, *, outputs_real_space=True, removes_padding=True,
             mask=None, filter=None, normalizes_signal=False, **kw):
    """AbstractImageModel.simulate.  base_image_model.py:68-105, 194-213."""
    fourier_image = compute_fourier_image(grid, frequency_slice, spec, **kw)
    if removes_padding:
        return postprocess(fourier_image, spec, outputs_real_space=outputs_real_space, mask=mask, filter=filter,
                           normalizes_signal=normalizes_signal)
    return irfftn(fourier_image, s=spec.padded_shape) if outputs_real_space else fourier_image


# ---------------------------------------------------------------------------
# Noise model and loss  (cryojax/simulator/_noise_model/gaussian_noise_model.py)
# ---------------------------------------------------------------------------


def white_noise_fourier(rng, padded_shape, variance, pixel_size):
    """Fourier-space white noise draw before postprocess: std*N(0,1), [0,0]=0.

    cryojax/simulator/_noise_model/gaussian_noise_model.py:167-205.
    """
    freqs = padded_frequency_grid_in_angstroms(padded_shape, pixel_size)
    std = np.sqrt(math.prod(padded_shape) * variance)
    noise = std * rng.standard_normal(freqs.shape[:-1])
    noise[0, 0] = 0.0
    return noise.astype(np.complex128)


def gaussian_white_log_likelihood(simulated, observed, variance):
    """cryojax/simulator/_noise_model/gaussian_noise_model.py:207-255."""
    r = simulated - observed
    return float(np.sum(-(np.abs(r) ** 2 / (2 * variance) + np.log(2 * np.pi * variance) / 2)))


def gaussian_colored_log_likelihood(simulated_fourier, observed_fourier, variance_grid, n_pixels):
    """cryojax/simulator/_noise_model/gaussian_noise_model.py:334-397: per-mode
    |r|^2 / (2 v) + log(2 pi v) / 2 with v = n_pixels * variance_fn(freqs), summed over
    the rfft half plane with column 0 (rows >= 1) once and the other columns twice,
    divided by n_pixels and negated."""
    v = n_pixels * np.asarray(variance_grid, np.float64)
    per_mode = np.abs(simulated_fourier - observed_fourier) ** 2 / (2 * v) + np.log(2 * np.pi * v) / 2
    return float(-(per_mode[1:, 0].sum() + 2 * per_mode[:, 1:].sum()) / n_pixels)


def normalize_image(image):
    """Zero mean, unit standard deviation.  cryojax/ndimage/_normalize.py:11-28."""
    return (image - image.mean()) / image.std()


def normalized_cross_correlation(simulated, observed):
    """Mean over pixels of normalize_image(sim) * normalize_image(obs) (Pearson r).

    The score of the pose-search benchmark: the zero-mean, unit-std real-space
    dot product (cryojax/ndimage/_normalize.py:11-28), divided by the pixel
    count so that it lies in [-1, 1].
    """
    return float(np.mean(normalize_image(simulated) * normalize_image(observed)))


def grid_search_orientations(grid, frequency_slice, specs, observed, quaternions, **kw):
    """Exhaustive orientation search: best (max NCC) grid index per image.

    For each image b, simulate spec b at every orientation of the grid (its
    own CTF, offsets and scale; the spec's wxyz is replaced) and keep the
    running best with the first index winning ties -- the elementwise
    running argmin of MinimumSearchMethod.batch_update applied to -NCC
    (cryojax/jax_util/_grid_search/search_method.py:237-265,
    search_loop.py:24-158).  Returns (best_index (n,), scores (n, T)).
    ``kw`` goes to compute_fourier_image (e.g. ``spline=True``).
    """
    import copy

    n, t = len(specs), len(quaternions)
    scores = np.empty((n, t))
    for b, spec in enumerate(specs):
        for k, q in enumerate(quaternions):
            s = copy.copy(spec)
            s.wxyz = np.asarray(q, np.float64)
            scores[b, k] = normalized_cross_correlation(simulate(grid, frequency_slice, s, **kw), observed[b])
    best = np.empty(n, np.int64)
    for b in range(n):
        cur, idx = np.inf, 0
        for k in range(t):  # strict "<" keeps the earliest index on ties
            if -scores[b, k] < cur:
                cur, idx = -scores[b, k], k
        best[b] = idx
    return best, scores


# ---------------------------------------------------------------------------
# Synthetic inputs (seeded): Gaussian-sum volumes, poses, CTF draws
# ---------------------------------------------------------------------------


def gaussian_sum_volume(box, n_gaussians, seed, *, centre_region=None, sigma_range=(1.0, 3.0),
                        amplitude_range=(0.5, 1.5), truncate=5.0):
    """Sum of isotropic 3-D Gaussians a*exp(-|r-c|^2/(2 sigma^2)) on a box^3 grid.

    Voxel coordinates are integer indices [z, y, x].  Centres are uniform in
    the cube [lo, hi)^3 where (lo, hi) = centre_region (default: the middle
    60 % of the box).  Each Gaussian is evaluated within +-truncate*sigma
    voxels of its centre (the synthetic volume's definition).
    """
    rng = np.random.default_rng(seed)
    if centre_region is None:
        centre_region = (0.2 * box, 0.8 * box)
    lo, hi = centre_region
    centres = rng.uniform(lo, hi, size=(n_gaussians, 3))
    sigmas = rng.uniform(sigma_range[0], sigma_range[1], size=n_gaussians)
    amps = rng.uniform(amplitude_range[0], amplitude_range[1], size=n_gaussians)
    vol = np.zeros((box, box, box), np.float64)
    for c, s, a in zip(centres, sigmas, amps):
        r = int(math.ceil(truncate * s))
        lo_i = np.maximum(np.floor(c).astype(int) - r, 0)
        hi_i = np.minimum(np.floor(c).astype(int) + r + 1, box)
        g = []
        for ax in range(3):
            x = np.arange(lo_i[ax], hi_i[ax], dtype=np.float64)
            g.append(np.exp(-((x - c[ax]) ** 2) / (2 * s * s)))
        vol[lo_i[0]:hi_i[0], lo_i[1]:hi_i[1], lo_i[2]:hi_i[2]] += (
            a * g[0][:, None, None] * g[1][None, :, None] * g[2][None, None, :]
        )
    return vol


def uniform_poses(n, seed, max_offset):
    """n uniform SO(3) quaternions (Shoemake) and x/y offsets ~ U(-max_offset, max_offset)."""
    rng = np.random.default_rng(seed)
    u1 = rng.uniform(0.0, 1.0, n)
    u2 = rng.uniform(0.0, 2 * np.pi, n)
    u3 = rng.uniform(0.0, 2 * np.pi, n)
    q = sample_uniform_quaternion(u1, u2, u3)
    offsets = rng.uniform(-max_offset, max_offset, size=(n, 2))
    return q, offsets


def relative_l2(a, b):
    """||a - b|| / ||b|| (b is the float64 reference)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))
