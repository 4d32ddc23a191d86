"""GPU: what the trained pose-proposal network gains over the search without it.

A small version of the pose-search benchmark (64^3 volume padded to 128^3,
64^2 images at SNR 0.1, a 192-direction x 24 in-plane grid = 4,608
orientations): the network is trained on the device by its own kernels,
then

* the learned search (top-8 directions x 24 in-plane = 192 candidates, 24x
  fewer than exhaustive) must agree with the exhaustive optimum on >= 90 %
  of the images before any fallback, while the same budget of random
  directions (the method without the network) agrees on far fewer;
* with the fallback threshold calibrated on separate images, agreement
  must reach >= 97 % with at most a third of the images falling back.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(cuda_device):
    import torch

    from cryojax_b200 import pose_training as PT
    from cryojax_b200 import simulator as S
    from cryojax_b200 import synthetic as Y
    from cryojax_b200.healpix import OrientationGrid
    from cryojax_b200.pose_net import PoseProposalNet

    vol = Y.gaussian_sum_volume(64, 300, 11)
    V = S.FourierVoxelGridVolume.from_real_voxel_grid(torch.as_tensor(vol, device="cuda"), pad_scale=2.0)
    cfg = S.BasicImageConfig((64, 64), 2.0, 300.0)
    grid = OrientationGrid(nside=4, n_inplane=24)
    data = PT.TrainingSet(V, cfg, 40000, seed=1, nside=4)
    net = PoseProposalNet(64, grid.n_dir, max_batch=256, seed=0)
    hist = PT.train_pose_net(net, data, epochs=10, lr=1e-3, snr=0.1, snr_start=2.0, snr_ramp=0.6)
    assert hist["loss"][-1] < 0.6 * hist["loss"][0]
    return V, cfg, grid, net


def _batch(V, cfg, n, seed, snr):
    import torch

    from cryojax_b200 import rotations as rot
    from cryojax_b200 import simulator as S
    from cryojax_b200.pose_training import simulate_clean_images

    rng = np.random.default_rng(seed)
    q = rot.sample_uniform_quaternions(rng, n)
    df = rng.uniform(8000, 20000, n)
    clean = simulate_clean_images(V, cfg, q, df)
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    noisy = clean + torch.randn(clean.shape, generator=g, device="cuda") * torch.sqrt(
        clean.var(dim=(1, 2), keepdim=True) / snr)
    ctf = S.AstigmaticCTF(defocus_in_angstroms=df, astigmatism_in_angstroms=np.zeros(n), astigmatism_angle=np.zeros(n))
    tt = S.ContrastTransferTheory(ctf, amplitude_contrast_ratio=0.1)
    model = S.make_image_model(V, cfg, S.QuaternionPose(np.zeros(n), np.zeros(n), wxyz=q), tt)
    return model, noisy


def test_learned_proposals_beat_random_proposals(setup):
    import torch

    from cryojax_b200.search import LearnedPoseSearch, PoseSearch

    V, cfg, grid, net = setup
    model, noisy = _batch(V, cfg, 96, 5, 0.1)
    search = PoseSearch(grid.rotation_matrices())
    ex = search.run(model, noisy)
    learned = LearnedPoseSearch(net, grid, top_k=8, search=search).run(model, noisy, fallback=False)
    agree_learned = float(np.mean(learned.best_orientation == ex.best_orientation))
    rng = np.random.default_rng(0)
    dirs = np.stack([rng.choice(grid.n_dir, 8, replace=False) for _ in range(96)])
    cand = (dirs[:, :, None] * grid.n_inplane + np.arange(grid.n_inplane)).reshape(96, -1).astype(np.int32)
    rnd = search.run(model, noisy, candidates=torch.as_tensor(cand, device="cuda"))
    agree_random = float(np.mean(rnd.best_orientation == ex.best_orientation))
    assert agree_learned >= 0.90, agree_learned
    assert agree_random <= 0.25, agree_random
    # learned candidates are a subset of the grid: never a better score than exhaustive
    assert np.all(learned.best_score <= ex.best_score + 1e-6)


def test_calibrated_fallback_reaches_agreement(setup):
    from cryojax_b200.search import LearnedPoseSearch, PoseSearch

    V, cfg, grid, net = setup
    search = PoseSearch(grid.rotation_matrices())
    cal_model, cal_noisy = _batch(V, cfg, 128, 7, 0.1)
    cal_ex = search.run(cal_model, cal_noisy)
    ls = LearnedPoseSearch(net, grid, top_k=8, search=search)
    thr = ls.calibrate_threshold(cal_model, cal_noisy, cal_ex.best_orientation, target_agreement=1.0)
    assert np.isfinite(thr)  # the fallback is always live: at least the least confident 2 % fall back
    model, noisy = _batch(V, cfg, 256, 9, 0.1)
    ex = search.run(model, noisy)
    res = ls.run(model, noisy)
    agree = float(np.mean(res.best_orientation == ex.best_orientation))
    assert agree >= 0.99, (agree, res.fallback.mean(), thr)
    assert 0 < res.fallback.mean() <= 1 / 3, res.fallback.mean()
    # fallback images carry the exhaustive answer exactly
    np.testing.assert_array_equal(res.best_orientation[res.fallback], ex.best_orientation[res.fallback])


def test_template_row_scoring_matches_simulated_candidates(setup):
    """The learned search with candidates scored from the shared template rows (cjx_ncc_directions) and the
    8 best re-ranked in FP32 returns the simulate-every-candidate answer on >= 99 % of the images (exactly
    whenever that answer is among the 8), and its FP16 candidate scores equal the template-sharing
    exhaustive search's scores of the same templates."""
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200.gradients import observed_to_fourier
    from cryojax_b200.search import LearnedPoseSearch, PoseSearch, TemplateSharingSearch

    V, cfg, grid, net = setup
    model, noisy = _batch(V, cfg, 128, 13, 0.1)
    search = PoseSearch(grid.rotation_matrices())
    shared = TemplateSharingSearch(grid.rotation_matrices(), rerank="simulate")
    sim = LearnedPoseSearch(net, grid, top_k=8, search=search).run(model, noisy, fallback=False)
    tmpl = LearnedPoseSearch(net, grid, top_k=8, search=search, templates=shared, rerank_top=8).run(
        model, noisy, fallback=False)
    agree = float(np.mean(sim.best_orientation == tmpl.best_orientation))
    assert agree >= 0.99, agree
    same = sim.best_orientation == tmpl.best_orientation
    np.testing.assert_array_equal(sim.best_score[same], tmpl.best_score[same])
    # the re-ranking from the FP32 template bank (the default): the same answers, scores to FP32 rounding
    bank = LearnedPoseSearch(net, grid, top_k=8, search=search, templates=TemplateSharingSearch(
        grid.rotation_matrices()), rerank_top=8).run(model, noisy, fallback=False)
    agree_b = float(np.mean(bank.best_orientation == tmpl.best_orientation))
    assert agree_b >= 0.99, agree_b
    same_b = bank.best_orientation == tmpl.best_orientation
    np.testing.assert_allclose(bank.best_score[same_b], tmpl.best_score[same_b], rtol=1e-5, atol=1e-7)

    # FP16 candidate sums against the exhaustive template GEMM's scores of the same templates
    obs_f = observed_to_fourier(noisy)
    pd = torch.as_tensor(model.image_params(), device="cuda")
    full = shared.run(model, obs_f, observed_is_fourier=True, image_params_device=pd, return_scores=True).scores
    dirs = tmpl.proposed_directions
    y16, z16, oo, yinv, zinv = shared._pack_observed(model, obs_f, pd)
    py, px = cfg.padded_shape
    kp = py * (px // 2 + 1)
    n, kd, ni = dirs.shape[0], dirs.shape[1], grid.n_inplane
    num = torch.empty((n, kd * ni), dtype=torch.float32, device="cuda")
    den = torch.empty_like(num)
    ws = torch.empty(nat.ncc_directions_workspace_size(n, kd, grid.n_dir), dtype=torch.uint8, device="cuda")
    nat.ncc_directions(y16, z16, shared.s16, shared.p16, kp, dirs, grid.n_dir, ni, num, den, ws)
    score = num * yinv[:, None] / torch.sqrt(den * zinv[:, None] * oo[:, None])
    t = (dirs.long()[:, :, None] * ni + torch.arange(ni, device="cuda")).reshape(n, -1)
    ref = full.gather(1, t)
    torch.testing.assert_close(score, ref, rtol=2e-3, atol=2e-4)
