"""Replica bookkeeping for multi-GPU runs.

The post-filter path has no data exchange: frames and streams are
independent, so N GPUs run N independent replicas (one process per GPU under
torchrun).  The only collectives are outside the data path: a barrier around
the timed region and one MAX reduction of the elapsed time.
"""
from __future__ import annotations


def max_over_ranks(value: float, device=None) -> float:
    """MAX of a scalar over the default process group (identity without one)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_mpixels(world: int, steps: int, pixels_per_step: int, elapsed_ms: float) -> float:
    """Whole-job Mpixel/s: every rank processed `steps` frames in at most `elapsed_ms`."""
    return world * steps * pixels_per_step / (elapsed_ms / 1e3) / 1e6


def frame_seeds(rank: int, count: int, config: int):
    """Distinct frame seeds per replica, so replicas never share inputs."""
    from .synth import seed_for

    return [seed_for(config, 100 * rank + i) for i in range(count)]
