"""Multi-GPU replicas of the chain: events shard by rank with no exchange
between ranks (the chain has no cross-event step), one process per GPU.

Only the job-level bookkeeping lives here: which events a rank processes,
and the job's rate from the per-rank device times (the slowest rank bounds
the job).  It runs over any torch.distributed backend: NCCL on the GPUs,
gloo in the CPU tests.
"""


def shard_seeds(rank, world, n_per_rank, base):
    """Seeds of the n_per_rank events rank `rank` processes: disjoint across
    ranks, so that the job's events are all distinct (weak scaling)."""
    if not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    return [base + rank * n_per_rank + k for k in range(n_per_rank)]


def job_rate(events_per_rank, ms_local, device=None):
    """(events/s of the whole job, max ms over ranks): every rank's events
    over the slowest rank's time.  Collective: every rank must call it.
    Without an initialised process group it is the local rate."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return events_per_rank / (ms_local / 1e3), ms_local
    world = dist.get_world_size()
    t = torch.tensor([float(ms_local)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    return world * events_per_rank / (ms / 1e3), ms
