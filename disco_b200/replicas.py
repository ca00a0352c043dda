"""Replicas across GPUs: one process per GPU, each advancing its own batch of
independent disks.

The reference's serial path is one domain on one processor, and the ragged
workload's disks are independent, so N GPUs run N replicas with no data-path
collective: every rank gets the same disk sizes with its own noise seeds
(fixed work per GPU, weak scaling), the ranks meet at a barrier around the
timed region, and the job's time is the maximum over ranks.  These are the
pieces bench.py uses; they are written against torch.distributed so that the
same code runs over NCCL on GPUs and over gloo on CPU (the tests).
"""


def rank_specs(rank, ndisk=64, seed=314159):
    """(Num_R, Mach_Number, noise seed) of each disk of `rank`: the sizes do
    not depend on the rank, the seeds do (ragged workload)."""
    from .workloads import ragged_specs
    return ragged_specs(ndisk, seed, rank)


def max_over_ranks(x, dist=None, device="cpu"):
    """The maximum of a per-rank float over all ranks (the rank itself when
    there is no process group)."""
    if dist is None or not dist.is_initialized():
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, units_per_rank, steps, max_ms):
    """Units processed by all ranks per second, timed by the slowest rank."""
    return world * units_per_rank * steps / (max_ms / 1e3)
