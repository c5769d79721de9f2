"""Replica timing over ranks for ``bench.py --gpus N`` (one process per GPU).

The reference fans independent outer batches over devices with no collective on the data
path (lib/mri/batch_sense.cpp:47-79); here every rank solves its own replica of the
workload (weak scaling), seeded per rank, and the only collectives are the barriers around
the timed region and the maximum of the ranks' step times.  The job's rate counts every
rank's units over that maximum."""
from __future__ import annotations

import torch


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Maximum of a per-rank float over the default process group; the value itself when
    there is no group or one rank.  ``device`` is where the reduction tensor lives (a CUDA
    device for NCCL, None = CPU for gloo)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, units_per_rank: float, ms_max: float) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time (ms)."""
    return world * float(units_per_rank) / (float(ms_max) / 1000.0)


def replica_seed(base: int, rank: int) -> int:
    """Seed of a rank's replica data: ranks solve different images of the same sizes."""
    return int(base) + 1000 * int(rank)
