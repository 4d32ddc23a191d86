"""HEALPix pixel centres (RING scheme) and the pose-search orientation grid.

Pixel centres follow the RING-scheme pix2ang formulas of Gorski et al.,
"HEALPix: a framework for high-resolution discretization and fast analysis
of data distributed on the sphere", ApJ 622:759 (2005), section 4: N_pix =
12 N_side^2 equal-area pixels on iso-latitude rings; polar-cap pixels
(p < N_cap = 2 N_side (N_side - 1)) sit on ring i with z = 1 - i^2 / (3
N_side^2), equatorial pixels on z = 4/3 - 2 i / (3 N_side), and the south cap
mirrors the north.

The reference samples orientations at random (SO3.sample_uniform,
cryojax/rotations/_lie_group.py:320-341); the grid here is the structured
grid of the pose-search benchmark.  An orientation (direction d = (theta,
phi), in-plane angle alpha) is the zyz Euler pose phi_angle = alpha,
theta_angle = theta, psi_angle = phi (cryojax/simulator/_pose.py:203-280):
its rotation R = Rz(phi) Ry(theta) Rz(alpha) has R[:, 2] = d, so the
slice plane (spanned by R[:, 0], R[:, 1]) is normal to d.
"""

from __future__ import annotations

import numpy as np

from . import rotations as rot


def _isqrt(v):
    r = np.floor(np.sqrt(np.asarray(v, np.float64))).astype(np.int64)
    # correct floating-point rounding of the square root
    r = np.where((r + 1) * (r + 1) <= v, r + 1, r)
    r = np.where(r * r > v, r - 1, r)
    return r


def pix2ang_ring(nside: int, pix=None):
    """(theta, phi) in radians of RING pixels (default: all 12 nside^2)."""
    npix = 12 * nside * nside
    ncap = 2 * nside * (nside - 1)
    p = np.arange(npix, dtype=np.int64) if pix is None else np.asarray(pix, np.int64)
    z = np.empty(p.shape, np.float64)
    phi = np.empty(p.shape, np.float64)
    north = p < ncap
    south = p >= npix - ncap
    eq = ~(north | south)
    # north polar cap
    pn = p[north]
    i = (1 + _isqrt(1 + 2 * pn)) >> 1
    j = (pn + 1) - 2 * i * (i - 1)
    z[north] = 1.0 - i * i / (3.0 * nside * nside)
    phi[north] = (j - 0.5) * np.pi / (2.0 * i)
    # equatorial belt
    pe = p[eq] - ncap
    i = pe // (4 * nside) + nside
    j = pe % (4 * nside) + 1
    fodd = np.where(((i + nside) & 1) == 1, 1.0, 0.5)
    z[eq] = (2 * nside - i) * 2.0 / (3.0 * nside)
    phi[eq] = (j - fodd) * np.pi / (2.0 * nside)
    # south polar cap
    ps = npix - p[south]
    i = (1 + _isqrt(2 * ps - 1)) >> 1
    j = 4 * i + 1 - (ps - 2 * i * (i - 1))
    z[south] = -1.0 + i * i / (3.0 * nside * nside)
    phi[south] = (j - 0.5) * np.pi / (2.0 * i)
    return np.arccos(np.clip(z, -1.0, 1.0)), phi


def pixel_directions(nside: int) -> np.ndarray:
    """Unit vectors (12 nside^2, 3) of the RING pixel centres."""
    theta, phi = pix2ang_ring(nside)
    st = np.sin(theta)
    return np.stack([st * np.cos(phi), st * np.sin(phi), np.cos(theta)], -1)


def nearest_pixel(nside: int, directions: np.ndarray) -> np.ndarray:
    """Index of the pixel centre closest to each unit vector (n, 3)."""
    centres = pixel_directions(nside)
    d = np.asarray(directions, np.float64).reshape(-1, 3)
    out = np.empty(d.shape[0], np.int64)
    for s in range(0, d.shape[0], 65536):
        out[s:s + 65536] = np.argmax(d[s:s + 65536] @ centres.T, axis=1)
    return out


class OrientationGrid:
    """n_dir = 12 nside^2 HEALPix directions x n_inplane in-plane angles.

    Orientation index o = direction * n_inplane + in-plane index.
    """

    def __init__(self, nside: int = 8, n_inplane: int = 48):
        self.nside = nside
        self.n_inplane = n_inplane
        self.theta, self.phi = pix2ang_ring(nside)
        self.n_dir = self.theta.size
        self.inplane_deg = np.arange(n_inplane) * (360.0 / n_inplane)

    @property
    def size(self) -> int:
        return self.n_dir * self.n_inplane

    def euler_angles(self, index=None) -> np.ndarray:
        """(n, 3) zyz Euler angles (phi, theta, psi) in degrees."""
        o = np.arange(self.size) if index is None else np.asarray(index, np.int64)
        d, a = o // self.n_inplane, o % self.n_inplane
        return np.stack([self.inplane_deg[a], np.rad2deg(self.theta[d]), np.rad2deg(self.phi[d])], -1)

    def quaternions(self, index=None) -> np.ndarray:
        e = self.euler_angles(index)
        return rot.euler_zyz_to_quat(e[:, 0], e[:, 1], e[:, 2])

    def rotation_matrices(self, index=None) -> np.ndarray:
        return rot.quat_to_matrix(self.quaternions(index))

    def direction_of(self, rotations: np.ndarray) -> np.ndarray:
        """HEALPix direction index nearest to each rotation's slice normal R[:, 2]."""
        R = np.asarray(rotations, np.float64).reshape(-1, 3, 3)
        return nearest_pixel(self.nside, R[:, :, 2])
