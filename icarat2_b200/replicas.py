"""Throughput of independent replicas, one process per GPU.

The designs of different GPUs share no data, so the data path has no
collective: each rank runs its own design loop and times it on its own
device with CUDA events.  The job took as long as its slowest rank and
processed the units of every rank, so the one collective is a max over ranks
of the per-rank totals (torch.distributed, NCCL on GPUs; gloo on CPU)."""


def job_rate(local_ms, units, world=1, dist=None, device=None):
    """(units per second of the whole job, the slowest rank's milliseconds)
    when every one of `world` ranks processed `units` units in local_ms."""
    import torch

    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    if ms <= 0.0:
        raise ValueError("non-positive timed region")
    return world * units / (ms / 1000.0), ms
