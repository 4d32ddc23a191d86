"""Host-side SO(3) helpers (float64, batched over leading axes).

These build the per-image rotation matrices passed to the kernels.  The
formulas are those of cryoJAX's SO3 (quaternions w, x, y, z, Hamilton
product):
  compose      cryojax/rotations/_lie_group.py:103-115
  inverse      cryojax/rotations/_lie_group.py:117-119
  as_matrix    cryojax/rotations/_lie_group.py:221-232
  exp          cryojax/rotations/_lie_group.py:234-271
  normalize    cryojax/rotations/_lie_group.py:316-318
  sample_uniform cryojax/rotations/_lie_group.py:320-341
For a unit quaternion, SO3.apply(v) = q (0, v) q^-1 equals as_matrix(q) @ v.
"""

from __future__ import annotations

import numpy as np


def quat_compose(q0, q1):
    q0 = np.asarray(q0, np.float64)
    q1 = np.asarray(q1, np.float64)
    w0, x0, y0, z0 = np.moveaxis(q0, -1, 0)
    w1, x1, y1, z1 = np.moveaxis(q1, -1, 0)
    return np.stack(
        [
            w0 * w1 - x0 * x1 - y0 * y1 - z0 * z1,
            w0 * x1 + x0 * w1 + y0 * z1 - z0 * y1,
            w0 * y1 - x0 * z1 + y0 * w1 + z0 * x1,
            w0 * z1 + x0 * y1 - y0 * x1 + z0 * w1,
        ],
        axis=-1,
    )


def quat_inverse(q):
    return np.asarray(q, np.float64) * np.array([1.0, -1.0, -1.0, -1.0])


def quat_normalize(q):
    q = np.asarray(q, np.float64)
    return q / np.linalg.norm(q, axis=-1, keepdims=True)


def quat_to_matrix(q):
    """Rotation matrix of q / |q| (batched)."""
    q = np.asarray(q, np.float64)
    norm = np.sum(q * q, axis=-1, keepdims=True)
    q = q * np.sqrt(2.0 / norm)
    w, x, y, z = np.moveaxis(q, -1, 0)
    return np.stack(
        [
            np.stack([1.0 - y * y - z * z, x * y - z * w, x * z + y * w], -1),
            np.stack([x * y + z * w, 1.0 - x * x - z * z, y * z - x * w], -1),
            np.stack([x * z - y * w, y * z + x * w, 1.0 - x * x - y * y], -1),
        ],
        axis=-2,
    )


def so3_exp(tangent):
    """Exponential map, tangent (..., 3) in radians -> quaternion (..., 4)."""
    t = np.asarray(tangent, np.float64)
    th2 = np.sum(t * t, axis=-1)
    th4 = th2 * th2
    taylor = th2 < 1e-10
    safe = np.sqrt(np.where(taylor, 1.0, th2))
    real = np.where(taylor, 1.0 - th2 / 8.0 + th4 / 384.0, np.cos(0.5 * safe))
    imag = np.where(taylor, 0.5 - th2 / 48.0 + th4 / 3840.0, np.sin(0.5 * safe) / safe)
    return np.concatenate([real[..., None], imag[..., None] * t], axis=-1)


def euler_zyz_to_quat(phi, theta, psi):
    """Extrinsic zyz Euler angles in degrees -> quaternion R3 @ R2 @ R1.

    cryojax/simulator/_pose.py:257-272.
    """
    phi, theta, psi = np.broadcast_arrays(*(np.deg2rad(np.asarray(a, np.float64)) for a in (phi, theta, psi)))
    z = np.zeros_like(phi)
    r1 = so3_exp(np.stack([z, z, phi], -1))
    r2 = so3_exp(np.stack([z, theta, z], -1))
    r3 = so3_exp(np.stack([z, z, psi], -1))
    return quat_compose(quat_compose(r3, r2), r1)


def sample_uniform_quaternions(rng: np.random.Generator, n: int):
    """n uniform rotations (Shoemake's S^3 sampling, same formula as the reference)."""
    u1 = rng.uniform(0.0, 1.0, n)
    u2 = rng.uniform(0.0, 2 * np.pi, n)
    u3 = rng.uniform(0.0, 2 * np.pi, n)
    a = np.sqrt(1.0 - u1)
    b = np.sqrt(u1)
    return np.stack([a * np.sin(u2), a * np.cos(u2), b * np.sin(u3), b * np.cos(u3)], -1)


def matrix_to_quat(R):
    """Unit quaternions (w, x, y, z) of rotation matrices (..., 3, 3), w >= 0.

    Shepperd's method (S. W. Shepperd, "Quaternion from rotation matrix",
    J. Guidance and Control 1, 1978): take the square root of the largest of
    4 w^2, 4 x^2, 4 y^2, 4 z^2 from the trace and diagonal, then the other
    components from the off-diagonal sums and differences.
    """
    R = np.asarray(R, np.float64)
    shp = R.shape[:-2]
    R = R.reshape(-1, 3, 3)
    tr = R[:, 0, 0] + R[:, 1, 1] + R[:, 2, 2]
    cand = np.stack([1 + tr, 1 + 2 * R[:, 0, 0] - tr, 1 + 2 * R[:, 1, 1] - tr, 1 + 2 * R[:, 2, 2] - tr], -1)
    k = np.argmax(cand, axis=1)
    q = np.empty((R.shape[0], 4))
    s = np.sqrt(np.maximum(cand[np.arange(len(k)), k], 0.0))  # = 2 |component k|
    for idx in range(4):
        m = k == idx
        if not np.any(m):
            continue
        r, ss = R[m], s[m]
        if idx == 0:
            q[m] = np.stack([ss / 2, (r[:, 2, 1] - r[:, 1, 2]) / (2 * ss), (r[:, 0, 2] - r[:, 2, 0]) / (2 * ss),
                             (r[:, 1, 0] - r[:, 0, 1]) / (2 * ss)], -1)
        elif idx == 1:
            q[m] = np.stack([(r[:, 2, 1] - r[:, 1, 2]) / (2 * ss), ss / 2, (r[:, 0, 1] + r[:, 1, 0]) / (2 * ss),
                             (r[:, 0, 2] + r[:, 2, 0]) / (2 * ss)], -1)
        elif idx == 2:
            q[m] = np.stack([(r[:, 0, 2] - r[:, 2, 0]) / (2 * ss), (r[:, 0, 1] + r[:, 1, 0]) / (2 * ss), ss / 2,
                             (r[:, 1, 2] + r[:, 2, 1]) / (2 * ss)], -1)
        else:
            q[m] = np.stack([(r[:, 1, 0] - r[:, 0, 1]) / (2 * ss), (r[:, 0, 2] + r[:, 2, 0]) / (2 * ss),
                             (r[:, 1, 2] + r[:, 2, 1]) / (2 * ss), ss / 2], -1)
    q *= np.where(q[:, :1] < 0, -1.0, 1.0)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q.reshape(shp + (4,))
