"""GPU: pipeline.HostStreamingSimulator (pinned host parameters in, pinned host images out, two streams).

Its images must be the device path's images bit for bit (each image's kernels are independent of the
sub-batching, of the orientation order inside a sub-batch and of the stream), and the device path is
pinned against the float64 oracle at rel-L2 <= 1e-5.  The sub-batch plan ramps sub_batch / 8, / 4, / 2
before full sub-batches and covers every image exactly once.
"""

import numpy as np
import pytest

from oracle import cryojax_oracle as O
from tests.helpers import IMAGE_REL_L2_TOL, make_volume, random_specs, rel_l2_per_image, specs_to_model_args

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,sub_batch", [(37, 16), (300, 64), (5, 2048)])
def test_host_streaming_matches_device_path(cuda_device, n, sub_batch):
    import torch

    from cryojax_b200 import simulator as S
    from cryojax_b200.pipeline import HostStreamingSimulator

    _, grid, fs = make_volume(32, 60, seed=n)
    specs = random_specs(n, seed=n + 1, shape=(32, 32))
    pose, tt, cfg = specs_to_model_args(specs)
    vol = S.FourierVoxelGridVolume(torch.as_tensor(grid.astype(np.complex64)).cuda())
    model = S.make_image_model(vol, cfg, pose, tt)
    direct = model.compute_fourier_image().cpu().numpy()

    sim = HostStreamingSimulator(vol, cfg, model.volume_integrator, model._flags(), sub_batch=sub_batch)
    plan = sim.sub_batches(n)
    assert sum(c for _, c in plan) == n and [s for s, _ in plan] == list(np.cumsum([0] + [c for _, c in plan])[:-1])
    assert all(c <= sub_batch for _, c in plan)
    ph = sim.pinned_params(model.image_params())
    oh = sim.pinned_output(n)
    for _ in range(2):  # a second call reuses the streams' buffers
        sim.run(ph, oh)
        torch.cuda.synchronize()
        assert np.array_equal(oh.numpy(), direct)

    ref = np.stack([O.compute_fourier_image(grid, fs, s) for s in specs[:8]])
    assert max(rel_l2_per_image(oh.numpy()[:8], ref)) <= IMAGE_REL_L2_TOL
