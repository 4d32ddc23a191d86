"""GPU: simulate_particle_stack from the reference's RELION STAR fixture through the batched device launch.

The particles of tests/golden/relion/test_starfile.star (16^2 images at
12 A, their own poses, defoci, astigmatism and envelope) are simulated with
one device call per batch, written to an MRC stack, read back, and compared
with the float64 oracle fed the same STAR rows through the reference's
conversions (defocus = (U + V) / 2, astigmatism = U - V, pose =
EulerAnglePose(-originX, -originY, -rot, -tilt, -psi)).  Tolerance: rel-L2
per image IMAGE_REL_L2_TOL (1e-5); the float32 MRC storage adds ~1e-7.
"""

import os
import shutil

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import IMAGE_REL_L2_TOL, make_volume, rel_l2_per_image

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "relion")


def _oracle_specs(pf):
    d = pf.starfile_data["particles"]
    o = pf.starfile_data["optics"].iloc[0]
    specs = []
    for _, r in d.iterrows():
        specs.append(O.ImageSpec(
            shape=(int(o["rlnImageSize"]),) * 2, pixel_size=float(o["rlnImagePixelSize"]),
            voltage_in_kilovolts=float(o["rlnVoltage"]),
            wxyz=O.euler_pose_quaternion(-r["rlnAngleRot"], -r["rlnAngleTilt"], -r["rlnAnglePsi"]),
            offset_in_angstroms=np.array([-r["rlnOriginXAngst"], -r["rlnOriginYAngst"]]),
            defocus_in_angstroms=0.5 * (r["rlnDefocusU"] + r["rlnDefocusV"]),
            astigmatism_in_angstroms=r["rlnDefocusU"] - r["rlnDefocusV"], astigmatism_angle=r["rlnDefocusAngle"],
            spherical_aberration_in_mm=float(o["rlnSphericalAberration"]),
            amplitude_contrast_ratio=float(o["rlnAmplitudeContrast"]), phase_shift=r["rlnPhaseShift"],
            envelope_b_factor=r["rlnCtfBfactor"], envelope_amplitude=r["rlnCtfScalefactor"]))
    return specs


@pytest.mark.parametrize("batch_size", [None, 2])
def test_simulate_particle_stack_from_the_fixture_star_file(cuda_device, tmp_path, batch_size):
    import torch

    from cryojax_b200 import relion
    from cryojax_b200 import simulator as S

    shutil.copyfile(os.path.join(HERE, "test_starfile.star"), tmp_path / "in.star")
    pf = relion.RelionParticleParameterFile(tmp_path / "in.star", loads_envelope=True)
    specs = _oracle_specs(pf)
    _, grid, fs = make_volume(16, 30, seed=12, pad_scale=2.0)
    volume = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())

    out = relion.RelionParticleParameterFile(tmp_path / "out" / "sim.star", mode="w", loads_envelope=True)
    out.append(pf[:])  # the same parameters in a new project
    ds = relion.RelionParticleStackDataset(out, tmp_path / "out", mode="w")

    def compute(parameters, vol, _):
        model = S.make_image_model(vol, parameters["image_config"], parameters["pose"], parameters["transfer_theory"])
        return model.simulate()

    relion.simulate_particle_stack(ds, compute, constant_args=volume, batch_size=batch_size)
    back = relion.RelionParticleStackDataset(
        relion.RelionParticleParameterFile(tmp_path / "out" / "sim.star", loads_envelope=True), tmp_path / "out")
    got = back[:]["images"]
    ref = np.stack([O.simulate(grid, fs, s) for s in specs])
    assert got.shape == ref.shape == (3, 16, 16)
    errs = rel_l2_per_image(got, ref)
    assert max(errs) <= IMAGE_REL_L2_TOL, errs
