"""Multi-GPU by replicas: one process per GPU, each analysing its own video
(the path shards by video with no data exchange). The only collective is the
timing reduction: the whole-job time of a step is the slowest rank's, and the
whole-job throughput is the frames all ranks processed over that time."""


def rank_seed(base, rank):
    """Each rank's video seed (distinct, reproducible)."""
    return base + rank


def max_over_ranks(value, dist=None, device="cpu"):
    """MAX all-reduce of a scalar across the process group (identity without one)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_throughput(units_per_rank, ms_per_step_max, world):
    """Units per second of the whole job: every rank processed
    units_per_rank per step, the step took the slowest rank's time."""
    return world * units_per_rank / (ms_per_step_max / 1e3)
