"""RELION STAR / MRC I/O against the reference's own fixtures and known answers (CPU).

Fixtures: tests/golden/relion/test_starfile.star and 000000.mrcs, byte
copies of cryojax tests/data (written by tests/golden/make_fixtures.py).
The expected values restate cryojax tests/test_relion_dataset.py:181-470
(CTF, pose, inverse pose, envelope, optics broadcasting, pad options) and
its write / append / numbering behaviour; round trips are exact for the
STAR columns (6 decimals) and the float32 MRC data.
"""

import os
import shutil

import numpy as np
import pytest

from cryojax_b200 import mrc, relion, star
from cryojax_b200 import simulator as S

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "relion")
STAR = os.path.join(HERE, "test_starfile.star")


@pytest.fixture
def project(tmp_path):
    shutil.copyfile(os.path.join(HERE, "000000.mrcs"), tmp_path / "000000.mrcs")
    shutil.copyfile(STAR, tmp_path / "particles.star")
    return tmp_path


def test_star_reader_reads_the_fixture():
    d = star.read_starfile(STAR)
    assert set(d) == {"particles", "optics"}
    p, o = d["particles"], d["optics"]
    assert p.shape == (3, 16) and o.shape == (1, 6)
    assert p["rlnClassNumber"].dtype == np.int64 and p["rlnDefocusU"].dtype == np.float64
    assert p["rlnImageName"].tolist() == ["0000001@000000.mrcs", "0000002@000000.mrcs", "0000003@000000.mrcs"]
    assert float(p["rlnDefocusU"][0]) == 10061.054688 and int(o["rlnImageSize"][0]) == 16


def test_mrc_reader_reads_the_fixture_stack():
    a = mrc.read_array_from_mrc(os.path.join(HERE, "000000.mrcs"))
    assert a.shape == (3, 16, 16) and a.dtype == np.float64
    h = mrc.read_mrc_header(os.path.join(HERE, "000000.mrcs"))
    assert (h["nx"], h["ny"], h["nz"], h["mode"], h["ispg"]) == (16, 16, 3, 2, 0)
    np.testing.assert_allclose(a.mean(), h["dmean"], rtol=1e-5)


def test_ctf_and_pose_params():
    pf = relion.RelionParticleParameterFile(STAR, loads_envelope=False, loads_metadata=True)
    p = pf[:]
    ctf, tt, pose = p["transfer_theory"].ctf, p["transfer_theory"], p["pose"]
    data = pf.starfile_data["particles"]
    u, v = data["rlnDefocusU"].to_numpy(), data["rlnDefocusV"].to_numpy()
    np.testing.assert_allclose(ctf.defocus_in_angstroms, 0.5 * (u + v), rtol=1e-12)
    np.testing.assert_allclose(ctf.astigmatism_in_angstroms, u - v, rtol=1e-12)
    np.testing.assert_allclose(ctf.astigmatism_angle, data["rlnDefocusAngle"], rtol=1e-12)
    np.testing.assert_allclose(tt.phase_shift, data["rlnPhaseShift"])
    np.testing.assert_allclose(ctf.spherical_aberration_in_mm, 2.7)
    np.testing.assert_allclose(tt.amplitude_contrast_ratio, 0.1)
    assert tt.envelope is None
    np.testing.assert_allclose(pose.offset_in_angstroms[:, 0], -data["rlnOriginXAngst"])
    np.testing.assert_allclose(pose.offset_in_angstroms[:, 1], -data["rlnOriginYAngst"])
    np.testing.assert_allclose(pose.phi_angle, -data["rlnAngleRot"])
    np.testing.assert_allclose(pose.theta_angle, -data["rlnAngleTilt"])
    np.testing.assert_allclose(pose.psi_angle, -data["rlnAnglePsi"])
    # one particle: scalar parameters
    p0 = pf[0]
    assert np.ndim(p0["transfer_theory"].ctf.defocus_in_angstroms) == 0
    assert p0["metadata"] is not None and "rlnClassNumber" in p0["metadata"].columns
    assert "rlnDefocusU" not in p0["metadata"].columns


def test_inverse_rotation_is_the_inverse():
    a = relion.RelionParticleParameterFile(STAR, inverts_rotation=False)[:]["pose"]
    b = relion.RelionParticleParameterFile(STAR, inverts_rotation=True)[:]["pose"]
    qa, qb = a.quaternion(), b.quaternion()
    qb = qb * np.sign(qb[:, :1] * qa[:, :1])  # q and -q are the same rotation
    np.testing.assert_allclose(qa * np.array([1, -1, -1, -1]), qb, atol=1e-12)
    np.testing.assert_allclose(a.rotation_matrices(), np.swapaxes(b.rotation_matrices(), -1, -2), atol=1e-12)


def test_envelope_broadcasting_and_pad_options():
    pf = relion.RelionParticleParameterFile(STAR, loads_envelope=True, pad_options=dict(shape=(22, 22)))
    p = pf[:]
    env = p["transfer_theory"].envelope
    np.testing.assert_allclose(env.b_factor, 1.0)
    np.testing.assert_allclose(env.amplitude, 2.0)
    assert p["image_config"].shape == (16, 16) and p["image_config"].padded_shape == (22, 22)
    assert p["image_config"].pixel_size.shape == (3,)
    pf.broadcasts_image_config = False
    assert np.ndim(pf[:]["image_config"].pixel_size) == 0
    # selection
    sel = relion.RelionParticleParameterFile(STAR, selection_filter={"rlnAngleRot": lambda x: x > 100.0})
    assert len(sel) == 2
    with pytest.raises(IndexError):
        pf[5]


def test_stack_dataset_reads_images(project):
    pf = relion.RelionParticleParameterFile(project / "particles.star")
    ds = relion.RelionParticleStackDataset(pf, project)
    ref = mrc.read_array_from_mrc(project / "000000.mrcs")
    out = ds[:]
    np.testing.assert_array_equal(out["images"], ref)
    assert out["parameters"]["pose"].batch_size == 3
    np.testing.assert_array_equal(ds[1]["images"], ref[1])
    ds.loads_parameters = False
    assert ds[np.array([2, 0])]["parameters"] is None
    np.testing.assert_array_equal(ds[np.array([2, 0])]["images"], ref[[2, 0]])


def _params(n, seed):
    rng = np.random.default_rng(seed)
    pose = S.EulerAnglePose(rng.uniform(-5, 5, n), rng.uniform(-5, 5, n), rng.uniform(-180, 180, n),
                            rng.uniform(0, 180, n), rng.uniform(-180, 180, n))
    ctf = S.AstigmaticCTF(rng.uniform(8000, 20000, n), rng.uniform(0, 400, n), rng.uniform(0, 180, n), 2.7)
    tt = S.ContrastTransferTheory(ctf, envelope=S.FourierGaussian(rng.uniform(0.5, 1.5, n), rng.uniform(10, 90, n)),
                                  amplitude_contrast_ratio=0.07, phase_shift=rng.uniform(0, 30, n))
    cfg = S.BasicImageConfig((24, 24), 1.5, 300.0)
    return {"image_config": cfg, "pose": pose, "transfer_theory": tt}


def test_write_append_and_read_back(tmp_path):
    pf = relion.RelionParticleParameterFile(tmp_path / "out.star", mode="w")
    ds = relion.RelionParticleStackDataset(pf, tmp_path / "proj", mode="w",
                                           mrcfile_settings=dict(prefix="f", output_folder="stacks"))
    p1, p2 = _params(4, 1), _params(3, 2)
    rng = np.random.default_rng(3)
    im1, im2 = rng.standard_normal((4, 24, 24)), rng.standard_normal((3, 24, 24))
    ds.append({"parameters": p1, "images": im1})
    ds.append({"parameters": p2, "images": im2})
    names = pf.starfile_data["particles"]["rlnImageName"].tolist()
    assert names[0] == "000001@stacks/f_000000.mrcs" and names[4] == "000001@stacks/f_000001.mrcs"
    assert pf.starfile_data["optics"]["rlnOpticsGroup"].tolist() == [1, 2]
    pf.save()
    with pytest.raises(FileExistsError):
        pf.save()
    back = relion.RelionParticleParameterFile(tmp_path / "out.star", loads_envelope=True)
    r = back[np.arange(0, 4)]
    np.testing.assert_allclose(r["pose"].phi_angle, p1["pose"].phi_angle, atol=1e-6)
    np.testing.assert_allclose(r["pose"].offset_in_angstroms, p1["pose"].offset_in_angstroms, atol=1e-6)
    np.testing.assert_allclose(r["transfer_theory"].ctf.defocus_in_angstroms, p1["transfer_theory"].ctf.defocus_in_angstroms,
                               atol=1e-6)
    np.testing.assert_allclose(r["transfer_theory"].ctf.astigmatism_in_angstroms,
                               p1["transfer_theory"].ctf.astigmatism_in_angstroms, atol=2e-6)
    np.testing.assert_allclose(r["transfer_theory"].envelope.b_factor, p1["transfer_theory"].envelope.b_factor, atol=1e-6)
    np.testing.assert_allclose(r["transfer_theory"].amplitude_contrast_ratio, 0.07)
    rd = relion.RelionParticleStackDataset(back, tmp_path / "proj", loads_parameters=False)
    np.testing.assert_array_equal(rd[0:4]["images"], im1.astype(np.float32))
    np.testing.assert_array_equal(rd[np.array([4, 6])]["images"], im2[[0, 2]].astype(np.float32))
    with pytest.raises(NotImplementedError):  # two optics groups in one read
        back[:]


def test_set_item_updates_rows(tmp_path):
    shutil.copyfile(STAR, tmp_path / "p.star")
    pf = relion.RelionParticleParameterFile(tmp_path / "p.star")
    new = _params(1, 5)
    pf[1] = {"pose": S.EulerAnglePose(1.0, 2.0, 10.0, 20.0, 30.0), "transfer_theory": new["transfer_theory"]}
    row = pf.starfile_data["particles"].iloc[1]
    assert (row["rlnOriginXAngst"], row["rlnAngleTilt"]) == (-1.0, -20.0)
    assert pf[1]["pose"].theta_angle == 20.0


def test_simulate_particle_stack_control_flow(tmp_path):
    pf = relion.RelionParticleParameterFile(tmp_path / "s.star", mode="w")
    pf.append(_params(7, 9))
    ds = relion.RelionParticleStackDataset(pf, tmp_path / "proj", mode="w")
    calls = []

    def fn(parameters, constant, per_particle):
        n = parameters["pose"].batch_size or 1
        calls.append(n)
        out = np.zeros((n, 24, 24)) + constant + np.asarray(per_particle, float).reshape(n, 1, 1)
        return out if parameters["pose"].batch_size else out[0]

    relion.simulate_particle_stack(ds, fn, constant_args=1.0, per_particle_args=np.arange(7.0), batch_size=3,
                                   images_per_file=5)
    assert calls == [3, 2, 2]  # files of 5 and 2 images, batches of at most 3
    back = relion.RelionParticleStackDataset(relion.RelionParticleParameterFile(tmp_path / "s.star"), tmp_path / "proj")
    imgs = back[:]["images"]
    np.testing.assert_array_equal(imgs[:, 0, 0], 1.0 + np.arange(7.0))
    assert back.parameter_file.starfile_data["particles"]["rlnImageName"].tolist()[5] == "000001@000001.mrcs"
    with pytest.raises(ValueError):
        relion.simulate_particle_stack(back, fn)


def test_mrc_round_trips(tmp_path):
    rng = np.random.default_rng(0)
    v = rng.standard_normal((8, 10, 12)).astype(np.float32)
    mrc.write_volume_to_mrc(v, 1.25, tmp_path / "v.mrc")
    got, d = mrc.read_array_from_mrc(tmp_path / "v.mrc", loads_grid_spacing=True)
    np.testing.assert_array_equal(got, v)
    assert d == 1.25 and mrc.read_mrc_header(tmp_path / "v.mrc")["ispg"] == 1
    mrc.write_image_to_mrc(v[0], 2.0, tmp_path / "i.mrc")
    assert mrc.read_array_from_mrc(tmp_path / "i.mrc").shape == (10, 12)
    with pytest.raises(FileExistsError):
        mrc.write_image_to_mrc(v[0], 2.0, tmp_path / "i.mrc")
    with pytest.raises(OSError):
        mrc.write_image_stack_to_mrc(v, 2.0, tmp_path / "s.mrc")


def test_star_edge_cases(tmp_path):
    p = tmp_path / "e.star"
    p.write_text("# comment\n\ndata_general\n\n_rlnImageSize 64\n_rlnComment 'two words'\n\n"
                 "data_particles\n\nloop_\n_rlnA #1\n_rlnName #2\n1\t\"a b\"\n2\tc\n\n")
    d = star.read_starfile(p)
    assert d["general"]["rlnImageSize"].tolist() == [64]
    assert d["particles"]["rlnName"].tolist() == ["a b", "c"] and d["particles"]["rlnA"].dtype == np.int64
    star.write_starfile(d, tmp_path / "o.star")
    back = star.read_starfile(tmp_path / "o.star")
    assert back["particles"]["rlnName"].tolist() == ["a b", "c"]
    bad = tmp_path / "bad.star"
    bad.write_text("data_x\nloop_\n_rlnA #1\n_rlnB #2\n1 2 3\n")
    with pytest.raises(ValueError):
        star.read_starfile(bad)
    with pytest.raises(OSError):
        star.read_starfile(tmp_path / "x.txt")


def test_mrc_big_endian_and_modes(tmp_path):
    import struct

    data = np.arange(2 * 3 * 4, dtype=">i2").reshape(2, 3, 4)
    header = bytearray(1024)
    struct.pack_into(">10i", header, 0, 4, 3, 2, 1, 0, 0, 0, 4, 3, 2)
    struct.pack_into(">3f", header, 40, 8.0, 6.0, 4.0)
    struct.pack_into(">2i", header, 88, 1, 0)
    header[208:212] = b"MAP "
    header[212:216] = b"\x11\x11\x00\x00"
    (tmp_path / "be.mrc").write_bytes(bytes(header) + data.tobytes())
    got, d = mrc.read_array_from_mrc(tmp_path / "be.mrc", loads_grid_spacing=True)
    np.testing.assert_array_equal(got, data.astype(np.float64))
    assert d == 2.0
    (tmp_path / "short.mrc").write_bytes(bytes(header) + data.tobytes()[:10])
    with pytest.raises(ValueError):
        mrc.read_array_from_mrc(tmp_path / "short.mrc")


def test_mrc_header_statistics_match_numpy_float64():
    """The writer's header min / max / mean / rms against NumPy in float64 (header fields are float32)."""
    from cryojax_b200.mrc import _header_stats

    rng = np.random.default_rng(3)
    for shape, offset in [((3, 5), 0.0), ((40, 64, 64), 100.0), ((2, 1000, 1001), -7.5)]:
        a = (rng.standard_normal(shape) * 3 + offset).astype(np.float32)
        lo, hi, mean, rms = _header_stats(a)
        assert lo == float(a.min()) and hi == float(a.max())
        np.testing.assert_allclose(mean, a.mean(dtype=np.float64), rtol=1e-6, atol=1e-7)
        np.testing.assert_allclose(rms, a.std(dtype=np.float64), rtol=1e-6)
    assert _header_stats(np.zeros((0, 4), np.float32)) == (0.0, 0.0, 0.0, 0.0)
