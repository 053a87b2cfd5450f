"""Multi-GPU host logic: one process per GPU, particles sharded by rank, geometry replicated, no data-path collective.

Every rank evaluates its own particle set over the same (small, static) geometry: the path has no exchange step, so a
run on N GPUs is N independent shards (weak scaling: the per-rank work is fixed as N grows).  The only collectives are
the barrier around the timed region and the max over ranks of the measured time; serving scales by replicas.
"""
import numpy as np
import torch
import torch.distributed as dist


def rank_particles(n, rank, base, box=4.0):
    """the particle set of `rank`: rank 0 keeps `base` (the reference workload's own particles), the others draw n
    seeded uniform positions in [0, box]^2 (seed 1000 + rank)."""
    if rank == 0:
        return base
    return np.random.default_rng(1000 + rank).uniform(0, box, size=(n, 2))


def max_over_ranks(value, device=None):
    """the largest `value` over all ranks (the device time of a step is the slowest rank's); `value` without a
    process group."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, device=None):
    """the sum of `value` over all ranks (the units of the whole job); `value` without a process group."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(units_per_rank, seconds, world):
    """whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return units_per_rank * world / seconds
