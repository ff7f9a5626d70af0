"""Multi-GPU rendering: one process per GPU over torch.distributed.

Paths are independent, so the work shards by sample index with no exchange while rendering:
rank r renders samples [r * spp_per_rank, (r + 1) * spp_per_rank) of a world * spp_per_rank-sample
image (every (pixel, sample) path keeps the PCG32 stream the single-GPU render would give it,
because the stream is seeded by pixel * total_spp + sample).  The job's one exchange is the
final combination of the per-rank Welford images: a count-weighted mean, as one all-reduce of
mean x count plus one of the counts (NCCL over NVLink on GPUs, gloo on CPU).  The scene, BVH and
environment are replicated per rank.
"""
from __future__ import annotations


def sample_range(rank: int, world: int, spp_per_rank: int) -> tuple[int, int]:
    """(first sample, sample count) of `rank` in a world * spp_per_rank-sample render."""
    if not (0 <= rank < world) or spp_per_rank <= 0:
        raise ValueError("bad rank / world / spp_per_rank")
    return rank * spp_per_rank, spp_per_rank


def combine(mean, count, group=None):
    """Count-weighted mean of the per-rank images: sum(mean_r * count_r) / sum(count_r).

    mean: torch tensor (H, W, C) (this rank's running mean), count: int or tensor broadcastable
    to mean's leading dims.  Returns the combined image on every rank."""
    import torch
    import torch.distributed as dist

    c = torch.as_tensor(count, dtype=mean.dtype, device=mean.device)
    while c.dim() < mean.dim():
        c = c.unsqueeze(-1)
    acc = mean * c
    tot = c.expand_as(mean[..., :1]).clone()
    dist.all_reduce(acc, group=group)
    dist.all_reduce(tot, group=group)
    return acc / tot
