"""Shared helpers for the parity tests: seeded inputs and oracle comparisons."""

from __future__ import annotations

import numpy as np

from oracle import cryojax_oracle as O

# Floating-point tolerance of the FP32 kernels against the float64 oracle:
# relative L2 error per image (||gpu - oracle|| / ||oracle||).
IMAGE_REL_L2_TOL = 1e-5


def make_volume(box, n_gaussians, seed, pad_scale=2.0, sigma_range=(1.0, 2.5)):
    vol = O.gaussian_sum_volume(box, n_gaussians, seed, sigma_range=sigma_range)
    grid, fs = O.fourier_voxel_grid_from_real_voxel_grid(vol, pad_scale=pad_scale)
    return vol, grid, fs


def random_specs(n, seed, shape, padded_shape=None, pixel_size=2.0, max_offset=10.0, offset_z=False,
                 envelope=False):
    rng = np.random.default_rng(seed)
    q, off = O.uniform_poses(n, seed + 1, max_offset)
    specs = []
    for b in range(n):
        o = off[b]
        if offset_z:
            o = np.array([o[0], o[1], rng.uniform(-300, 300)])
        specs.append(O.ImageSpec(
            shape=shape, padded_shape=padded_shape, pixel_size=pixel_size, voltage_in_kilovolts=300.0,
            wxyz=q[b], offset_in_angstroms=o,
            defocus_in_angstroms=rng.uniform(5000, 25000), astigmatism_in_angstroms=rng.uniform(0, 500),
            astigmatism_angle=rng.uniform(0, 180), spherical_aberration_in_mm=2.7,
            amplitude_contrast_ratio=0.1, phase_shift=rng.uniform(0, 10),
            envelope_b_factor=(rng.uniform(20, 80) if envelope else None), envelope_amplitude=1.0))
    return specs


def specs_to_model_args(specs):
    """Batched host-side pose / CTF / config objects matching a list of oracle specs."""
    from cryojax_b200 import simulator as S

    q = np.stack([s.wxyz for s in specs])
    off = np.stack([s.offset_in_angstroms for s in specs])
    kw = {}
    if off.shape[1] == 3:
        kw["offset_z_in_angstroms"] = off[:, 2]
    pose = S.QuaternionPose(off[:, 0], off[:, 1], wxyz=q, **kw)
    ctf = S.AstigmaticCTF(
        defocus_in_angstroms=np.array([s.defocus_in_angstroms for s in specs]),
        astigmatism_in_angstroms=np.array([s.astigmatism_in_angstroms for s in specs]),
        astigmatism_angle=np.array([s.astigmatism_angle for s in specs]),
        spherical_aberration_in_mm=np.array([s.spherical_aberration_in_mm for s in specs]))
    env = None
    if specs[0].envelope_b_factor is not None:
        env = S.FourierGaussian(amplitude=np.array([s.envelope_amplitude for s in specs]),
                                b_factor=np.array([s.envelope_b_factor for s in specs]))
    tt = S.ContrastTransferTheory(ctf, envelope=env,
                                  amplitude_contrast_ratio=np.array([s.amplitude_contrast_ratio for s in specs]),
                                  phase_shift=np.array([s.phase_shift for s in specs]))
    s0 = specs[0]
    cfg = S.BasicImageConfig(s0.shape, s0.pixel_size, s0.voltage_in_kilovolts,
                             pad_options=dict(shape=s0.padded_shape))
    return pose, tt, cfg


def rel_l2_per_image(got, ref):
    return [O.relative_l2(g, r) for g, r in zip(got, ref)]
