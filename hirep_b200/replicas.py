"""Replica runs on several GPUs (one process per GPU, torch.distributed).

The fermion operator of one lattice lives on one GPU (the single-GPU scope has
no halo exchange), so N GPUs run N independent replicas of the same workload.
There is no collective on the data path: the only collectives are the timing
reductions below, taken between the timed regions.
"""


def max_over_ranks(value, dist, device):
    """The maximum of a per-rank scalar over all ranks (the job's time is the slowest rank's)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, t_max_ms, world):
    """Whole-job throughput: the units every rank processed, over the slowest rank's time."""
    return world * units_per_rank / (t_max_ms * 1e-3)
