"""One process per GPU, images sharded across ranks, volume replicated.

The simulation path has no exchange step: each rank simulates its own
images against its own replica of the volume, so the only cross-rank
operations are a barrier around the timed region and a max-reduction of
the ranks' device times (the job's time is the slowest rank's).  These
helpers hold that logic so it can be exercised with the `gloo` backend on
CPU as well as `nccl` on GPUs.
"""

from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class RankInfo:
    rank: int
    world: int
    local_rank: int


def rank_info() -> RankInfo:
    """RANK / WORLD_SIZE / LOCAL_RANK from a torchrun-style environment (defaults: one rank)."""
    return RankInfo(int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                    int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, info: RankInfo, timeout_s: float = 300.0) -> None:
    """Join the process group when there is more than one rank (MASTER_ADDR / MASTER_PORT from the env)."""
    if info.world > 1:
        import torch.distributed as dist

        dist.init_process_group(backend, rank=info.rank, world_size=info.world,
                                timeout=datetime.timedelta(seconds=timeout_s))


def shutdown(info: RankInfo) -> None:
    if info.world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def image_seed(seed: int, rank: int) -> int:
    """Seed of a rank's own image batch: every rank draws different poses and CTFs."""
    return seed + 1 + 1000 * rank


def barrier(info: RankInfo) -> None:
    if info.world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(value_ms: float, info: RankInfo, device=None) -> float:
    """The largest of the ranks' values (a collective: every rank must call it)."""
    if info.world == 1:
        return float(value_ms)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: int, info: RankInfo, steps: int, job_ms: float) -> float:
    """Whole-job units/s: every rank's units over the slowest rank's time."""
    return units_per_rank * info.world * steps / (job_ms / 1000.0)
