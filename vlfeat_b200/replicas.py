"""Multi-GPU Fisher encoding as independent replicas (one process per GPU).

Images are independent, so N GPUs run N replicas, each on its own batch, with
no exchange on the data path (weak scaling).  The only collectives are the two
the measurement needs: the step time is the maximum over ranks (the job ends
when its slowest replica does), and the job's work is the sum of the ranks'
descriptors.  Both run over the process group the caller set up (NCCL on GPUs;
gloo in the CPU tests).
"""
from __future__ import annotations


def rank_data_seed(rank: int) -> int:
    """Seed of a rank's synthetic descriptors: every replica encodes its own data."""
    return 300 + int(rank)


def _tensor(value, dist):
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    return torch.tensor([float(value)], dtype=torch.float64, device=dev)


def max_over_ranks(value: float, dist) -> float:
    """The maximum of `value` over the ranks (every rank receives it)."""
    if dist is None:
        return float(value)
    t = _tensor(value, dist)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_units(units: float, dist) -> float:
    """The sum of the ranks' units of work (descriptors) in one step."""
    if dist is None:
        return float(units)
    t = _tensor(units, dist)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def whole_job_rate(units_per_rank: float, ms_per_rank: float, dist) -> tuple[float, float]:
    """(units per second of the whole job, the step time in ms): all ranks'
    units over the slowest rank's step time."""
    ms = max_over_ranks(ms_per_rank, dist)
    return job_units(units_per_rank, dist) / (ms / 1e3), ms
