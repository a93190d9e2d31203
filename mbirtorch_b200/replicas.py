"""Multi-GPU use of the path: independent replicas.

A reconstruction runs on one GPU with no sharding, so N GPUs serve N
independent jobs (one process per GPU) and share no data.  The ranks
exchange only their timings: a whole-job rate is the work of all ranks over
the slowest rank's time, taken on the device and reduced with MAX.
"""

import torch


def max_over_ranks(value, device=None):
    """The maximum of a per-rank float over the default process group (the
    value itself when there is no group or one rank)."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else 'cpu')
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, seconds_max, world):
    """Whole-job throughput of `world` replicas that each did
    `units_per_rank` units, the slowest in `seconds_max` seconds."""
    if seconds_max <= 0:
        raise ValueError('the slowest rank time must be positive')
    return world * units_per_rank / seconds_max
