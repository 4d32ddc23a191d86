"""Local refinement of orientation and defocus by gradient descent through
the adjoint kernels (cjx_slice_ctf_loss_grad).

For each image the loss is the squared residual between its simulation and
the observed image (the loss of the reference's README gradient example,
through LinearImageModel.simulate, cryojax/simulator/_image_model/
base_image_model.py:68-105, 297-328).  One refinement step is one call of
the loss + gradient kernels over the whole batch; every image then moves on
its own, alternating between the two parameter groups (rotation on odd
steps, defocus on even ones, so that a noisy step in one group never rides
on a good step in the other):

  rotation  R <- exp(-a w_hat) R, w_hat = g_w / |g_w|, with g_w = dL/dw the
            gradient for a left rotation exp(w) R, g_w = sum_j R[:, j] x
            dL/dR[:, j] over the two columns that span the slice plane;
  defocus   df <- df - b sign(dL/d df).

Step lengths a (radians) and b (Angstrom) adapt per image and group: a
step that lowers the loss is kept and that group's next step is 1.25x
longer; one that raises it is undone and the step halves.  After `steps`
evaluations (the first at the starting point) each image keeps the
lowest-loss point it has seen.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _native as nat
from . import rotations as rot
from .gradients import observed_to_fourier


def _torch():
    import torch

    return torch


@dataclass
class RefineResult:
    rotations: np.ndarray      # (n, 3, 3)
    defocus: np.ndarray        # (n,) Angstrom (including any out-of-plane offset)
    loss: np.ndarray           # (n,) final squared residual
    loss_history: np.ndarray   # (steps, n) loss of each evaluated point
    accepted: np.ndarray       # (n,) accepted steps


def _exp_so3(w):
    """Rotation matrices exp([w]x) (Rodrigues) for axis-angle vectors (n, 3)."""
    q = rot.so3_exp(w)
    return rot.quat_to_matrix(q)


def rotation_step_gradient(R, g, ewald=False):
    """dL/dw at w = 0 for the rotation step R -> exp([w]x) R, from the per-image gradient records g (n, 16):
    the sum over R's columns c of R[:, c] x dL/dR[:, c] (columns 0 and 1; column 2 too on the Ewald sphere,
    whose surface has a third coordinate)."""
    n = g.shape[0]
    dR = g[:, nat.G_ROT:nat.G_ROT + 6].reshape(n, 3, 2)
    gw = np.cross(R[:, :, 0], dR[:, :, 0]) + np.cross(R[:, :, 1], dR[:, :, 1])
    if ewald:
        gw = gw + np.cross(R[:, :, 2], g[:, nat.G_ROT + 6:nat.G_ROT + 9])
    return gw


def refine_poses(image_model, observed, *, steps=20, rot_step_deg=2.0, defocus_step=200.0, grow=1.25, shrink=0.5,
                 observed_is_fourier=False, min_rot_step_deg=1e-3, min_defocus_step=0.1) -> RefineResult:
    """Refine every image's rotation and defocus starting from the image model's pose and CTF.

    observed: real-space images (n, P, P) in cryoJAX's convention or their
    rfftn (``observed_is_fourier``).  Needs padded_shape == shape (the
    adjoint's condition).
    """
    torch = _torch()
    from .simulator import orientation_order

    cfg = image_model.image_config
    if tuple(cfg.padded_shape) != tuple(cfg.shape):
        raise NotImplementedError("refinement needs padded_shape == shape")
    vol = image_model.volume_parametrization.get_representation()
    integ = image_model.volume_integrator
    ewald = not integ.is_projection_approximation  # the surface's third coordinate: R's third column enters
    dev = vol.device
    params = image_model.image_params().copy()
    n = params.shape[0]
    flags = image_model._flags() | integ._base_flags()
    if hasattr(vol, "spline_coefficients"):  # FourierVoxelSplineVolume: cubic-spline samples and gradients
        flags |= nat.CJX_GRID_SPLINE | nat.CJX_GRID_BRICKED
        grid = vol.bricked_grid()
    else:  # the x-pair layout: 4 vector loads per sample in the forward and the scatter
        flags |= nat.CJX_GRID_BRICKED_PAIRS
        grid = vol.pair_grid()
    py, px = cfg.padded_shape
    desc = nat.make_desc(vol.shape[0], py, px, flags, integ.fill_value)
    obs_f = observed if observed_is_fourier else observed_to_fourier(observed)
    order = torch.as_tensor(orientation_order(params[:, 0:9].reshape(-1, 3, 3)), device=dev)
    pd = torch.empty((n, params.shape[1]), dtype=torch.float64, device=dev)
    grads = torch.empty((n, nat.GRAD_DOUBLES), dtype=torch.float64, device=dev)
    ws = torch.empty(max(nat.loss_workspace_size(desc, n), 1), dtype=torch.uint8, device=dev)

    cur = params.copy()
    best = params.copy()
    best_loss = np.full(n, np.inf)
    best_gw = np.zeros((n, 3))
    best_gdf = np.zeros(n)
    a = np.full(n, np.deg2rad(rot_step_deg))
    b = np.full(n, float(defocus_step))
    accepted = np.zeros(n, np.int64)
    hist = np.empty((steps, n))
    for it in range(steps):
        pd.copy_(torch.from_numpy(cur))
        nat.slice_ctf_loss_grad(desc, grid, pd, obs_f, grads, None, ws, order=order)
        g = grads.cpu().numpy()
        loss = g[:, nat.G_LOSS]
        hist[it] = loss
        gw = rotation_step_gradient(cur[:, 0:9].reshape(n, 3, 3), g, ewald)
        better = loss < best_loss
        if it > 0:
            accepted += better
            if it % 2 == 1:  # this evaluation tested a rotation step
                a = np.where(better, a * grow, np.maximum(a * shrink, np.deg2rad(min_rot_step_deg)))
            else:
                b = np.where(better, b * grow, np.maximum(b * shrink, min_defocus_step))
        best[better] = cur[better]
        best_loss[better] = loss[better]
        best_gw[better] = gw[better]
        best_gdf[better] = g[better, nat.G_DF]
        if it == steps - 1:
            break
        cur = best.copy()
        if (it + 1) % 2 == 1:  # next: a rotation step from each image's best point
            norm = np.linalg.norm(best_gw, axis=1, keepdims=True)
            w = -a[:, None] * best_gw / np.where(norm > 0, norm, 1.0)
            cur[:, 0:9] = (_exp_so3(w) @ best[:, 0:9].reshape(n, 3, 3)).reshape(n, 9)
        else:  # next: a defocus step
            cur[:, nat.P_DEFOCUS] = best[:, nat.P_DEFOCUS] - b * np.sign(best_gdf)
    return RefineResult(best[:, 0:9].reshape(n, 3, 3).copy(), best[:, nat.P_DEFOCUS].copy(), best_loss, hist,
                        accepted)


def rotation_angle_deg(Ra, Rb):
    """Angle (degrees) of Ra Rb^T for stacks of rotation matrices."""
    c = (np.einsum("nij,nij->n", np.asarray(Ra), np.asarray(Rb)) - 1.0) / 2.0
    return np.degrees(np.arccos(np.clip(c, -1.0, 1.0)))


def with_rotations_and_defocus(image_model, rotations, defocus):
    """A copy of a batched image model with new rotations (n, 3, 3) and defocus (n,)."""
    import copy

    from .simulator import QuaternionPose

    m = copy.copy(image_model)
    off = image_model.pose.offset_in_angstroms
    n = len(defocus)
    off = np.broadcast_to(off.reshape(-1, off.shape[-1]) if off.ndim > 1 else off, (n, off.shape[-1]))
    kw = {"offset_z_in_angstroms": off[:, 2]} if off.shape[-1] == 3 else {}
    m.pose = QuaternionPose(off[:, 0], off[:, 1], wxyz=rot.matrix_to_quat(np.asarray(rotations)), **kw)
    tt = copy.copy(image_model.transfer_theory)
    tt.ctf = copy.copy(tt.ctf)
    base = np.asarray(defocus, np.float64) - (off[:, 2] if off.shape[-1] == 3 else 0.0)
    tt.ctf.defocus_in_angstroms = base
    m.transfer_theory = tt
    return m
