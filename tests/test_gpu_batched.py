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
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            while not stop.is_set():
                got = models[1].compute_fourier_image()
                stream.synchronize()
                if not torch.equal(got, ref):
                    errors.append("images changed while the autotuner ran")
                if [nat.tuning_get(k) for k in knobs] != before:
                    errors.append("process knobs changed while the autotuner ran")

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
