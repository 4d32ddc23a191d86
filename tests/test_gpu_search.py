"""GPU: orientation search (cjx_search through the C-ABI) against the oracle's grid search.

The oracle simulates every (image, orientation) pair in float64 and scores
it with normalize_image semantics (Pearson r); its running argmin of -NCC
keeps the earliest index on ties.  Tolerances: every device score within
NCC_ABS_TOL of the oracle's; the device's best orientation equals the
oracle's wherever the oracle's top two scores differ by more than
2 * NCC_ABS_TOL, and otherwise scores within NCC_ABS_TOL of the maximum.
"""

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import make_volume, specs_to_model_args

pytestmark = pytest.mark.gpu

NCC_ABS_TOL = 5e-5


def _specs(n, seed, shape, quats):
    rng = np.random.default_rng(seed)
    out = []
    for b in range(n):
        out.append(O.ImageSpec(shape=shape, pixel_size=2.0, wxyz=quats[b],
                               offset_in_angstroms=rng.uniform(-4, 4, 2),
                               defocus_in_angstroms=rng.uniform(8000, 20000),
                               astigmatism_in_angstroms=rng.uniform(0, 300), astigmatism_angle=rng.uniform(0, 180)))
    return out


def _observed(grid, fs, specs, seed, snr):
    rng = np.random.default_rng(seed)
    obs = []
    for s in specs:
        img = O.simulate(grid, fs, s)
        if snr is not None:
            img = img + rng.standard_normal(img.shape) * np.sqrt(img.var() / snr)
        obs.append(img)
    return np.stack(obs)


def _model(grid, specs):
    import torch

    from cryojax_b200 import simulator as S

    pose, tt, cfg = specs_to_model_args(specs)
    vol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
    return S.make_image_model(vol, cfg, pose, tt)


def _check_best(best, ref_scores):
    for b in range(ref_scores.shape[0]):
        s = np.sort(ref_scores[b])[::-1]
        if s[0] - s[1] > 2 * NCC_ABS_TOL:
            assert best[b] == int(np.argmax(ref_scores[b])), b
        else:
            assert ref_scores[b, best[b]] >= s[0] - NCC_ABS_TOL, b


@pytest.mark.parametrize("box,shape,snr", [(32, (32, 32), None), (32, (32, 32), 0.5), (48, (64, 64), 0.2)])
def test_exhaustive_scores_match_oracle(cuda_device, box, shape, snr):
    from cryojax_b200.healpix import OrientationGrid
    from cryojax_b200.search import PoseSearch

    og = OrientationGrid(nside=1, n_inplane=8)  # 96 orientations
    quats = og.quaternions()
    _, grid, fs = make_volume(box, 40, seed=box + 1)
    rng = np.random.default_rng(box)
    true_idx = rng.choice(og.size, 3, replace=False)
    specs = _specs(3, box + 2, shape, quats[true_idx])
    obs = _observed(grid, fs, specs, box + 3, snr)
    ref_best, ref_scores = O.grid_search_orientations(grid, fs, specs, obs, quats)

    res = PoseSearch(og.rotation_matrices()).run(_model(grid, specs), obs, return_scores=True)
    got = res.scores.cpu().numpy()
    assert got.shape == ref_scores.shape
    err = np.abs(got - ref_scores).max()
    assert err <= NCC_ABS_TOL, err
    _check_best(res.best_orientation, ref_scores)
    np.testing.assert_allclose(res.best_score, got[np.arange(3), res.best_orientation], rtol=0, atol=0)
    if snr is None:  # noiseless images drawn at grid orientations: the search recovers them
        np.testing.assert_array_equal(res.best_orientation, true_idx)
        assert np.all(res.best_score > 0.999)


def test_candidate_lists_score_the_same_as_exhaustive(cuda_device):
    from cryojax_b200.healpix import OrientationGrid
    from cryojax_b200.search import PoseSearch

    og = OrientationGrid(nside=1, n_inplane=8)
    quats = og.quaternions()
    _, grid, fs = make_volume(32, 40, seed=7)
    specs = _specs(4, 8, (32, 32), quats[[5, 17, 40, 90]])
    obs = _observed(grid, fs, specs, 9, 1.0)
    search = PoseSearch(og.rotation_matrices())
    model = _model(grid, specs)
    full = search.run(model, obs, return_scores=True)
    rng = np.random.default_rng(3)
    cand = np.stack([rng.choice(og.size, 11, replace=False) for _ in range(4)]).astype(np.int32)
    cand[:, 0] = cand[:, 3]  # a repeated candidate must not change the result
    part = search.run(model, obs, candidates=cand, return_scores=True)
    fs_ = full.scores.cpu().numpy()
    np.testing.assert_array_equal(part.scores.cpu().numpy(), fs_[np.arange(4)[:, None], cand])
    for b in range(4):
        sc = fs_[b, cand[b]]
        top = sc.max()
        assert part.best_score[b] == top
        assert part.best_orientation[b] == cand[b][sc == top].min()


def test_search_rejects_bad_candidates(cuda_device):
    from cryojax_b200.healpix import OrientationGrid
    from cryojax_b200.search import PoseSearch

    og = OrientationGrid(nside=1, n_inplane=4)
    _, grid, fs = make_volume(32, 10, seed=1)
    specs = _specs(2, 2, (32, 32), og.quaternions()[[0, 1]])
    obs = _observed(grid, fs, specs, 3, None)
    with pytest.raises(ValueError):
        PoseSearch(og.rotation_matrices()).run(_model(grid, specs), obs, candidates=np.full((2, 3), og.size))


@pytest.mark.parametrize("shift,spline", [(0.0, False), (4.0, False), (4.0, True)])
def test_template_sharing_search_matches_plain_scores(cuda_device, shift, spline):
    """FP16 GEMM scores within 2e-3 of the plain FP32 scorer; same argmax unless near-tied
    (trilinear volumes, and a FourierVoxelSplineVolume for both searches)."""
    from cryojax_b200 import simulator as S
    from cryojax_b200.healpix import OrientationGrid
    from cryojax_b200.search import PoseSearch, TemplateSharingSearch

    og = OrientationGrid(nside=2, n_inplane=8)  # 384 orientations
    quats = og.quaternions()
    _, grid, fs = make_volume(48, 60, seed=21)
    rng = np.random.default_rng(4)
    specs = _specs(12, 5, (64, 64), quats[rng.choice(og.size, 12, replace=False)])
    for s in specs:
        s.offset_in_angstroms = rng.uniform(-shift, shift, 2)
    obs = _observed(grid, fs, specs, 6, 0.3)
    model = _model(grid, specs)
    if spline:
        vol = S.FourierVoxelSplineVolume.from_fourier_voxel_grid(model.volume_parametrization.get_representation())
        pose, tt, cfg = specs_to_model_args(specs)
        model = S.make_image_model(vol, cfg, pose, tt)
    plain = PoseSearch(og.rotation_matrices()).run(model, obs, return_scores=True)
    shared = TemplateSharingSearch(og.rotation_matrices(), template_chunk=100, image_chunk=5).run(
        model, obs, return_scores=True)
    a, b = plain.scores.cpu().numpy(), shared.scores.cpu().numpy()
    assert np.abs(a - b).max() <= 2e-3, np.abs(a - b).max()
    for k in range(12):
        srt = np.sort(a[k])[::-1]
        if srt[0] - srt[1] > 4e-3:
            assert shared.best_orientation[k] == plain.best_orientation[k]
        assert abs(shared.best_score[k] - b[k].max()) == 0


@pytest.mark.parametrize("rerank", ["simulate", "bank"])
def test_template_sharing_rerank_equals_plain_exhaustive(cuda_device, rerank):
    """FP16 top-8 per image rescored in FP32: the plain exhaustive answer and score, bit for bit when each
    candidate is simulated again; from the FP32 template bank, the same answer and the score within 1e-5."""
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200.healpix import OrientationGrid
    from cryojax_b200.search import PoseSearch, TemplateSharingSearch

    og = OrientationGrid(nside=2, n_inplane=8)
    quats = og.quaternions()
    _, grid, fs = make_volume(48, 60, seed=23)
    rng = np.random.default_rng(8)
    specs = _specs(10, 9, (64, 64), quats[rng.choice(og.size, 10, replace=False)])
    obs = _observed(grid, fs, specs, 10, 0.1)
    model = _model(grid, specs)
    plain = PoseSearch(og.rotation_matrices()).run(model, obs, return_scores=True)
    ts = TemplateSharingSearch(og.rotation_matrices(), rerank=rerank)
    rr = ts.run(model, obs, rerank_top=8, return_scores=True)
    np.testing.assert_array_equal(rr.best_orientation, plain.best_orientation)
    if rerank == "simulate":
        np.testing.assert_array_equal(rr.best_score, plain.best_score)
    else:
        np.testing.assert_allclose(rr.best_score, plain.best_score, rtol=1e-5, atol=1e-7)
    # the top-k indices are the k best FP16 scores, descending
    fp16_scores = rr.scores.cpu().numpy()
    top = rr.candidates.cpu().numpy()
    for b in range(10):
        ref = np.argsort(-fp16_scores[b], kind="stable")[:8]
        np.testing.assert_array_equal(np.sort(top[b]), np.sort(ref))
        assert np.all(np.diff(fp16_scores[b, top[b]]) <= 0)
    assert nat.device_status() == 0


@pytest.mark.parametrize("kv,layout", [(300.0, "pairs"), (20.0, "linear")])
def test_ewald_search_scores_match_oracle(cuda_device, kv, layout):
    """PoseSearch on EwaldSphereExtraction + ContrastTransferTheory against the oracle's grid search
    on the Ewald contrast (every pair simulated in float64); 20 kV gives a strongly curved surface."""
    import torch

    from cryojax_b200 import simulator as S
    from cryojax_b200.healpix import OrientationGrid
    from cryojax_b200.search import PoseSearch, TemplateSharingSearch

    og = OrientationGrid(nside=1, n_inplane=4)  # 48 orientations
    quats = og.quaternions()
    _, grid, fs = make_volume(32, 40, seed=61)
    rng = np.random.default_rng(62)
    true_idx = rng.choice(og.size, 2, replace=False)
    specs = [O.ImageSpec(shape=(32, 32), pixel_size=2.0, voltage_in_kilovolts=kv, wxyz=quats[t],
                         offset_in_angstroms=rng.uniform(-4, 4, 2), defocus_in_angstroms=rng.uniform(8000, 20000),
                         astigmatism_in_angstroms=rng.uniform(0, 300), astigmatism_angle=rng.uniform(0, 180),
                         amplitude_contrast_ratio=0.1, phase_shift=rng.uniform(0, 20)) for t in true_idx]
    obs = np.stack([O.simulate(grid, fs, s, ewald=True) for s in specs])
    _, ref_scores = O.grid_search_orientations(grid, fs, specs, obs, quats, ewald=True)

    pose, tt, cfg = specs_to_model_args(specs)
    vol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
    integ = S.EwaldSphereExtraction(use_bricked_layout=layout != "linear", pair_layout=layout == "pairs")
    model = S.make_image_model(vol, cfg, pose, tt, volume_integrator=integ)
    res = PoseSearch(og.rotation_matrices()).run(model, obs, return_scores=True)
    got = res.scores.cpu().numpy()
    assert got.shape == ref_scores.shape
    err = np.abs(got - ref_scores).max()
    assert err <= NCC_ABS_TOL, err
    _check_best(res.best_orientation, ref_scores)
    np.testing.assert_array_equal(res.best_orientation, true_idx)  # noiseless images at grid orientations
    with pytest.raises(NotImplementedError):
        TemplateSharingSearch(og.rotation_matrices()).run(model, obs)
