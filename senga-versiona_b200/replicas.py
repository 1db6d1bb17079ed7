"""Multi-GPU bookkeeping of the replica runs (one independent box per rank).

The path does not shard in this build: N GPUs advance N independent boxes
with no data-path collective. The only cross-rank steps are a barrier around
the timed region and the maximum of the per-rank times, so the whole-job
rate is the points all ranks updated divided by the slowest rank's time.
"""


def max_over_ranks(value, device="cpu"):
    """Maximum of a per-rank scalar over the process group (the value itself
    without an initialised group of more than one rank)."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(points_per_rank, substages, world, seconds):
    """Grid-point substage updates per second of the whole job."""
    return points_per_rank * substages * world / seconds
