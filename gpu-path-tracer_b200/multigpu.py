"""Host-side logic of multi-GPU rendering (one process per GPU, torch.distributed).

Samples are independent, so a frame shards without a data-path collective: every rank renders
the same frame on its own Philox subsequences, and the per-pixel accumulation buffers are summed
once per frame (the only exchange step). With N ranks the combined image holds N x spp samples
per pixel (weak scaling: the work per GPU stays fixed as N grows).
"""
from __future__ import annotations


def rank_rng_offset(rank: int, samples_per_frame: int) -> int:
    """Philox subsequence offset of a rank: ranks draw from disjoint subsequence ranges."""
    if rank < 0 or samples_per_frame <= 0:
        raise ValueError("rank must be >= 0 and samples_per_frame > 0")
    return rank * samples_per_frame


def combine_accumulation(accumulation, dist) -> None:
    """Sum the per-pixel accumulation buffers of all ranks in place (NCCL on GPUs, gloo on CPU)."""
    dist.all_reduce(accumulation, op=dist.ReduceOp.SUM)


def max_over_ranks(values, dist, device="cpu"):
    """Element-wise maximum over ranks of a list of floats (device times are reported as the max)."""
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def combined_samples_per_pixel(spp: int, world: int) -> int:
    return spp * world
