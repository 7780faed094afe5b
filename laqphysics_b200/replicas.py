"""Independent replicas across GPUs (no collective on the data path).

One propagation couples every (r1, r2, channel) in each H·psi and needs global dot
products each Krylov iteration, so a single instance stays on one GPU.  Independent
instances (pulse-parameter scans, batched pump-probe cases, finite-difference probes —
the reference runs them as Slurm array jobs) are sharded one-per-GPU; the only
cross-rank operations are the timing reduction and an optional host gather of results.
"""
import numpy as np


def shard(instances, rank, world):
    """Instances of this rank: instance i goes to rank i mod world."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError('rank must be in [0, world)')
    return [x for i, x in enumerate(instances) if i % world == rank]


def max_over_ranks(value, dist=None, device=None):
    """Largest value over all ranks (the slowest rank sets the job time)."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_root(array, dist=None, device=None):
    """Concatenate per-rank result arrays on every rank (host gather of spectra)."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return [np.asarray(array)]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, np.asarray(array))
    return out


def whole_job_rate(units_per_rank, seconds_max, world):
    """Aggregate throughput: all ranks' units over the slowest rank's time."""
    if seconds_max <= 0:
        raise ValueError('time must be positive')
    return world * units_per_rank / seconds_max
