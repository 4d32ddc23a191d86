"""GPU: several volumes / image shapes in one cjx_slice_ctf_forward_multi call (and its CUDA graph)."""

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import IMAGE_REL_L2_TOL, make_volume, random_specs, rel_l2_per_image, specs_to_model_args

pytestmark = pytest.mark.gpu

GROUPS = [(24, (24, 24), 5), (32, (32, 32), 7), (40, (40, 40), 4), (32, (64, 64), 3)]  # (box, shape, images)


def _models_and_refs():
    import torch

    from cryojax_b200 import simulator as S

    models, refs = [], []
    for gi, (box, shape, nimg) in enumerate(GROUPS):
        vol, grid, fs = make_volume(box, 40, seed=100 + gi)
        specs = random_specs(nimg, seed=200 + gi, shape=shape)
        pose, tt, cfg = specs_to_model_args(specs)
        dvol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
        models.append(S.make_image_model(dvol, cfg, pose, tt))
        refs.append(np.stack([O.compute_fourier_image(grid, fs, s) for s in specs]))
    return models, refs


@pytest.mark.parametrize("tuning", [None, {"ilp": 4, "tile": 2}, "auto"])
def test_batched_groups_match_oracle(cuda_device, tuning, tmp_path, monkeypatch):
    from cryojax_b200.batched import BatchedSimulator

    monkeypatch.setenv("CRYOJAX_B200_AUTOTUNE_CACHE", str(tmp_path / "autotune.json"))
    models, refs = _models_and_refs()
    sim = BatchedSimulator(models, tuning=tuning, autotune_kw=dict(n_sample=8, repeats=1))
    outs = sim.run()
    for got, ref in zip(outs, refs):
        assert max(rel_l2_per_image(got.cpu().numpy(), ref)) <= IMAGE_REL_L2_TOL
    if tuning == "auto":
        assert (tmp_path / "autotune.json").exists()


def test_batched_cuda_graph_replay(cuda_device):
    import torch

    from cryojax_b200.batched import BatchedSimulator

    models, refs = _models_and_refs()
    sim = BatchedSimulator(models, tuning=None)
    sim.capture()
    for o in sim.outputs:
        o.zero_()
    for _ in range(2):
        sim.replay()
    torch.cuda.synchronize()
    for got, ref in zip(sim.outputs, refs):
        assert max(rel_l2_per_image(got.cpu().numpy(), ref)) <= IMAGE_REL_L2_TOL


def test_multi_validates_all_groups_before_launching(cuda_device):
    import torch

    from cryojax_b200 import _native as nat

    out = torch.zeros((1, 16, 9), dtype=torch.complex64, device="cuda")
    grid = torch.zeros((16, 16, 16), dtype=torch.complex64, device="cuda")
    params = torch.as_tensor(nat.empty_params(1), device="cuda")
    good = {"desc": nat.make_desc(16, 16, 16, 0), "grid": grid, "params": params, "out": out, "n_images": 1}
    bad = dict(good, desc=nat.make_desc(16, 16, 16, 1 << 30))
    out.fill_(7.0)
    with pytest.raises(nat.CryojaxB200Error):
        nat.slice_ctf_forward_multi(nat.make_groups([good, bad]))
    torch.cuda.synchronize()
    assert torch.all(out == 7.0)  # nothing ran


def test_autotune_leaves_process_knobs_alone_while_another_thread_simulates(cuda_device, tmp_path, monkeypatch):
    """The autotuner times its candidates through per-call choices: while it runs on one thread, forward
    calls on another thread (process-default knobs) keep giving the same images, and the knobs are unchanged
    afterwards."""
    import threading

    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200.batched import autotune

    monkeypatch.setenv("CRYOJAX_B200_AUTOTUNE_CACHE", str(tmp_path / "autotune.json"))
    models, refs = _models_and_refs()
    knobs = (nat.CJX_TUNE_GATHER_ILP, nat.CJX_TUNE_GATHER_TILE, nat.CJX_TUNE_CHUNK_BYTES, nat.CJX_TUNE_GATHER_MODE)
    before = [nat.tuning_get(k) for k in knobs]
    ref = models[1].compute_fourier_image().clone()
    errors, stop = [], threading.Event()

    def simulate_repeatedly():
        try:
            stream = torch.cuda.Stream()
            with torch.cuda.stream(stream):
                while not stop.is_set():
                    got = models[1].compute_fourier_image()
                    stream.synchronize()
                    if not torch.equal(got, ref):
                        errors.append("images changed while the autotuner ran")
                    if [nat.tuning_get(k) for k in knobs] != before:
                        errors.append("process knobs changed while the autotuner ran")
        except Exception as e:  # a failure on this thread must fail the test
            errors.append(repr(e))

    t = threading.Thread(target=simulate_repeatedly)
    t.start()
    try:
        for m in models:
            autotune(m, n_sample=8, repeats=1, use_cache=False)
    finally:
        stop.set()
        t.join()
    assert not errors, errors[:3]
    assert [nat.tuning_get(k) for k in knobs] == before


RESIZE_GROUPS = [(32, (32, 32), 5), (48, (64, 32), 7), (64, (64, 64), 4), (80, (96, 64), 6)]  # (box, shape, images)


@pytest.mark.parametrize("workspace", ["one_wave", "several_waves", "too_small"])
def test_waves_match_groups_one_after_another(cuda_device, workspace):
    """CJX_TUNE_MULTI_WAVES: every pass launched once per wave for all groups gives the groups-in-turn
    images bit for bit and the oracle's within tolerance: with the default chunks (one wave), with one-image
    chunks and twice their workspace (several waves of ragged sizes), and with one-image chunks and exactly
    their workspace, where one image of every group does not fit at once and the call runs the groups in
    turn instead."""
    one_image_chunks = workspace != "one_wave"
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200 import simulator as S

    models, refs, groups = [], [], []
    for gi, (box, shape, nimg) in enumerate(RESIZE_GROUPS):
        vol, grid, fs = make_volume(box, 40, seed=300 + gi)
        specs = random_specs(nimg, seed=400 + gi, shape=shape)
        pose, tt, cfg = specs_to_model_args(specs)
        dvol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
        m = S.make_image_model(dvol, cfg, pose, tt)
        models.append(m)
        refs.append(np.stack([O.compute_fourier_image(grid, fs, s) for s in specs]))
        integ = m.volume_integrator
        dgrid, layout = integ.device_grid(dvol)
        py, px = cfg.padded_shape
        groups.append({"desc": nat.make_desc(dvol.shape[0], py, px, m._flags() | layout, 0.0,
                                             1 if one_image_chunks else 0),
                       "grid": dgrid, "params": torch.as_tensor(m.image_params(), device="cuda"),
                       "order": None, "out": torch.zeros((nimg, py, px // 2 + 1), dtype=torch.complex64,
                                                         device="cuda"),
                       "n_images": nimg})
    arr = nat.make_groups(groups)
    factor = 2 if workspace == "several_waves" else 1
    ws = torch.empty(max(factor * nat.multi_workspace_size(arr), 1), dtype=torch.uint8, device="cuda")
    old = nat.tuning_get(nat.CJX_TUNE_MULTI_WAVES)
    try:
        nat.tuning_set(nat.CJX_TUNE_MULTI_WAVES, 0)
        nat.slice_ctf_forward_multi(arr, ws)
        seq = [g["out"].clone() for g in groups]
        for g in groups:
            g["out"].zero_()
        nat.tuning_set(nat.CJX_TUNE_MULTI_WAVES, 1)
        nat.profile_enable(True)
        nat.slice_ctf_forward_multi(arr, ws)
        torch.cuda.synchronize()
        prof = nat.profile_read()
        nat.profile_enable(False)
    finally:
        nat.tuning_set(nat.CJX_TUNE_MULTI_WAVES, old)
    if workspace == "too_small":
        assert "k_front_wave" not in prof, prof
    else:
        assert "k_front_wave" in prof and "k_rows_wave" in prof and "k_tail_wave" in prof, prof
        waves = prof["k_front_wave"][0]
        assert (waves > 1) == one_image_chunks, waves
        assert prof["k_rows_wave"][0] == waves and prof["k_tail_wave"][0] == waves
    for g, s, ref in zip(groups, seq, refs):
        torch.testing.assert_close(g["out"], s, rtol=0, atol=0)
        assert max(rel_l2_per_image(g["out"].cpu().numpy(), ref)) <= IMAGE_REL_L2_TOL


def test_waves_fall_back_when_a_group_cannot_join(cuda_device):
    """A group without the resize stage (Py = Px = N) cannot take the wave kernels: the call runs the groups
    in turn instead, with the same images."""
    import torch

    from cryojax_b200 import _native as nat
    from cryojax_b200.batched import BatchedSimulator

    models, refs = _models_and_refs()  # includes a no-resize group
    old = nat.tuning_get(nat.CJX_TUNE_MULTI_WAVES)
    try:
        nat.tuning_set(nat.CJX_TUNE_MULTI_WAVES, 1)
        sim = BatchedSimulator(models, tuning=None)
        nat.profile_enable(True)
        outs = sim.run()
        torch.cuda.synchronize()
        prof = nat.profile_read()
        nat.profile_enable(False)
    finally:
        nat.tuning_set(nat.CJX_TUNE_MULTI_WAVES, old)
    assert "k_front_wave" not in prof
    for got, ref in zip(outs, refs):
        assert max(rel_l2_per_image(got.cpu().numpy(), ref)) <= IMAGE_REL_L2_TOL
