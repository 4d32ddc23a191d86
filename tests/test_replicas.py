"""CPU: the multi-rank path (one process per GPU, images sharded, no data collective) on gloo.

Two ranks join a gloo process group on 127.0.0.1, build their own image
batches, and reduce their (different) timings: both must see the slower
rank's time, the whole-job rate must count both ranks' images, and the two
ranks' batches must differ.
"""

import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from cryojax_b200 import replicas, synthetic

    info = replicas.rank_info()
    replicas.init("gloo", info, timeout_s=60)
    batch = synthetic.image_batch(64, replicas.image_seed(2024, info.rank))
    replicas.barrier(info)
    job_ms = replicas.max_over_ranks(100.0 + 50.0 * info.rank, info)
    rate = replicas.job_rate(64, info, 3, job_ms)
    np.savez(os.path.join(out_dir, f"r{rank}.npz"), wxyz=batch.wxyz, job_ms=job_ms, rate=rate)
    replicas.shutdown(info)


def test_two_gloo_ranks_shard_images_and_take_the_slowest_time(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    r0, r1 = (np.load(tmp_path / f"r{r}.npz") for r in range(2))
    assert float(r0["job_ms"]) == float(r1["job_ms"]) == 150.0
    assert float(r0["rate"]) == pytest.approx(64 * 2 * 3 / 0.15)
    assert not np.allclose(r0["wxyz"], r1["wxyz"])


def test_single_rank_needs_no_process_group():
    from cryojax_b200 import replicas

    info = replicas.RankInfo(0, 1, 0)
    replicas.init("gloo", info)
    assert replicas.max_over_ranks(12.5, info) == 12.5
    assert replicas.job_rate(10, info, 2, 1000.0) == 20.0
    replicas.shutdown(info)
