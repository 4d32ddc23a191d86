"""Gradients of the squared residual through the Fourier-slice + CTF path.

``squared_residual_and_grad(model, observed)`` gives, for every image b of a
batched image model, L_b = sum_pixels (simulate_b() - observed_b)^2 (the
loss of the reference's README gradient example) and its derivatives with
respect to the pose parameters, the in-plane offsets, the defocus and the
Fourier voxel grid.  In the reference this is
``eqx.filter_grad(loss)(model)`` through
cryojax/simulator/_image_model/base_image_model.py:68-105, 297-328.

The device computes dL/dR (rotation matrix columns that span the slice
plane), dL/d(shift), dL/d(defocus) and the trilinear scatter-add for the
grid (cjx_slice_ctf_loss_grad).  The last step, from dL/dR to the pose's own
parameters (quaternion through its normalisation, zyz Euler angles in
degrees, or an axis-angle vector), is a float64 autograd on the host.
Complex gradients are dL/dRe + i dL/dIm (jax.grad returns the conjugate).
"""

from __future__ import annotations

import numpy as np

from . import _native as nat


def _torch():
    import torch

    return torch


# ---- rotation matrices as torch functions (float64, host) ---------------


def _quat_to_matrix_t(q):
    torch = _torch()
    norm = torch.sum(q * q, dim=-1, keepdim=True)
    q = q * torch.sqrt(2.0 / norm)
    w, x, y, z = q.unbind(-1)
    return torch.stack(
        [
            torch.stack([1.0 - y * y - z * z, x * y - z * w, x * z + y * w], -1),
            torch.stack([x * y + z * w, 1.0 - x * x - z * z, y * z - x * w], -1),
            torch.stack([x * z - y * w, y * z + x * w, 1.0 - x * x - y * y], -1),
        ],
        dim=-2,
    )


def _quat_mul_t(a, b):
    torch = _torch()
    w0, x0, y0, z0 = a.unbind(-1)
    w1, x1, y1, z1 = b.unbind(-1)
    return torch.stack(
        [
            w0 * w1 - x0 * x1 - y0 * y1 - z0 * z1,
            w0 * x1 + x0 * w1 + y0 * z1 - z0 * y1,
            w0 * y1 - x0 * z1 + y0 * w1 + z0 * x1,
            w0 * z1 + x0 * y1 - y0 * x1 + z0 * w1,
        ],
        -1,
    )


def _exp_t(t):
    torch = _torch()
    th = torch.sqrt(torch.sum(t * t, -1, keepdim=True).clamp_min(1e-300))
    small = th < 1e-5
    real = torch.where(small, 1.0 - th * th / 8.0, torch.cos(0.5 * th))
    imag = torch.where(small, 0.5 - th * th / 48.0, torch.sin(0.5 * th) / th)
    return torch.cat([real, imag * t], -1)


def _pose_rotation_t(pose, params):
    """Rotation matrices (n, 3, 3) of `pose` as a differentiable function of `params`."""
    from .simulator import AxisAnglePose, EulerAnglePose, QuaternionPose

    torch = _torch()
    if isinstance(pose, QuaternionPose):
        return _quat_to_matrix_t(params)
    if isinstance(pose, EulerAnglePose):
        rad = params * (np.pi / 180.0)
        z = torch.zeros_like(rad[:, 0])
        r1 = _exp_t(torch.stack([z, z, rad[:, 0]], -1))
        r2 = _exp_t(torch.stack([z, rad[:, 1], z], -1))
        r3 = _exp_t(torch.stack([z, z, rad[:, 2]], -1))
        return _quat_to_matrix_t(_quat_mul_t(_quat_mul_t(r3, r2), r1))
    if isinstance(pose, AxisAnglePose):
        return _quat_to_matrix_t(_exp_t(params * (np.pi / 180.0)))
    raise TypeError(f"unsupported pose type {type(pose).__name__}")


def _pose_param_array(pose, n):
    from .simulator import AxisAnglePose, EulerAnglePose, QuaternionPose

    if isinstance(pose, QuaternionPose):
        a = np.broadcast_to(pose.wxyz.reshape(-1, 4), (n, 4))
        return a, "d_wxyz"
    if isinstance(pose, EulerAnglePose):
        a = np.stack(np.broadcast_arrays(pose.phi_angle, pose.theta_angle, pose.psi_angle), -1).reshape(-1, 3)
        return np.broadcast_to(a, (n, 3)), "d_euler_angles"
    if isinstance(pose, AxisAnglePose):
        return np.broadcast_to(pose.euler_vector.reshape(-1, 3), (n, 3)), "d_euler_vector"
    raise TypeError(f"unsupported pose type {type(pose).__name__}")


def observed_to_fourier(observed):
    """cryoJAX rfftn of real-space images (ifftshift, then rfft2): complex64 [n, Py, Px//2+1]."""
    torch = _torch()
    obs = observed if isinstance(observed, torch.Tensor) else torch.as_tensor(np.asarray(observed))
    if obs.dim() == 2:
        obs = obs[None]
    return nat.rfft2(obs.to(device="cuda", dtype=torch.float32))


def squared_residual_and_grad(model, observed, *, grid_grad: bool = True, observed_is_fourier: bool = False,
                              sort_orientations: bool = True):
    """Loss and gradients for every image of a batched LinearImageModel / ContrastImageModel.

    observed: real-space images [n, Py, Px] (cryoJAX's centred convention),
    or their rfftn when ``observed_is_fourier``.  Needs padded_shape == shape.

    Returns a dict with ``loss`` (n,), the pose gradient under the pose's own
    parameter name (``d_wxyz`` (n, 4), ``d_euler_angles`` (n, 3) in degrees,
    or ``d_euler_vector`` (n, 3)), ``d_offset`` (n, 2), ``d_defocus`` (n,),
    ``d_rotation`` (n, 3, 2) (dL/dR for R's first two columns; (n, 3, 3) on the
    Ewald sphere, whose surface has a third coordinate) and, with ``grid_grad``,
    ``d_grid`` (complex64, shape of the grid, summed over the images).
    Volume integrators: FourierSliceExtraction and EwaldSphereExtraction (with
    a ContrastTransferTheory).
    """
    torch = _torch()
    from .simulator import orientation_order

    cfg = model.image_config
    if tuple(cfg.padded_shape) != tuple(cfg.shape):
        raise NotImplementedError("the loss gradient needs padded_shape == shape")
    vol = model.volume_parametrization.get_representation()
    integ = model.volume_integrator
    params = model.image_params()
    n = params.shape[0]
    ewald = not integ.is_projection_approximation  # EwaldSphereExtraction: R's third column enters too
    dev = vol.device
    flags = model._flags() | integ._base_flags()
    if hasattr(vol, "spline_coefficients"):  # gradient with respect to the spline coefficients
        grid, grad_shape = vol.spline_coefficients, tuple(vol.spline_coefficients.shape)
        flags |= nat.CJX_GRID_SPLINE
        if integ.use_bricked_layout:
            grid = vol.bricked_grid()
            flags |= nat.CJX_GRID_BRICKED
    else:
        grad_shape = tuple(vol.shape)
        if grid_grad and integ.use_bricked_layout:
            # with the grid scatter, the bricked layout: the x-pair copy's faster gather does not make up for
            # the L2 room its twice larger reads take from the scatter's atomics
            grid, layout = vol.bricked_grid(), nat.CJX_GRID_BRICKED
        else:  # the layout the forward reads (x-pair bricked by default)
            grid, layout = integ.device_grid(vol)
        flags |= layout
    py, px = cfg.padded_shape
    desc = nat.make_desc(vol.shape[0], py, px, flags, integ.fill_value)
    obs_f = observed if observed_is_fourier else observed_to_fourier(observed)
    if tuple(obs_f.shape) != (n, py, px // 2 + 1):
        raise ValueError(f"observed has shape {tuple(obs_f.shape)}, expected {(n, py, px // 2 + 1)} in Fourier space")
    pd = torch.as_tensor(params, device=dev)
    order = None
    if sort_orientations:
        order = torch.as_tensor(orientation_order(params[:, 0:9].reshape(-1, 3, 3)), device=dev)
    grads = torch.empty((n, nat.GRAD_DOUBLES), dtype=torch.float64, device=dev)
    gg = torch.zeros(grad_shape, dtype=torch.complex64, device=dev) if grid_grad else None
    ws = torch.empty(max(nat.loss_workspace_size(desc, n), 1), dtype=torch.uint8, device=dev)
    nat.slice_ctf_loss_grad(desc, grid, pd, obs_f, grads, gg, ws, order=order)
    g = grads.cpu().numpy()
    d_rot = g[:, nat.G_ROT:nat.G_ROT + 6].reshape(n, 3, 2)
    if ewald:  # the third column's entries follow the first two columns'
        d_rot = np.concatenate([d_rot, g[:, nat.G_ROT + 6:nat.G_ROT + 9, None]], axis=2)
    # chain dL/dR -> pose parameters (float64 autograd on the host)
    pvals, pname = _pose_param_array(model.pose, n)
    p_t = torch.tensor(np.ascontiguousarray(pvals), dtype=torch.float64, requires_grad=True)
    R = _pose_rotation_t(model.pose, p_t)
    (R[:, :, 0:d_rot.shape[2]] * torch.as_tensor(d_rot)).sum().backward()
    out = {
        "loss": g[:, nat.G_LOSS].copy(),
        pname: p_t.grad.numpy().copy(),
        "d_offset": g[:, nat.G_TX:nat.G_TY + 1].copy(),
        "d_defocus": g[:, nat.G_DF].copy(),
        "d_rotation": d_rot,
    }
    if grid_grad:
        out["d_grid"] = gg
    return out
