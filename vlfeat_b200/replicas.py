"""Multi-GPU Fisher encoding as independent replicas (one process per GPU),
and EM with its rows sharded over ranks.

Images are independent, so N GPUs run N replicas, each on its own batch, with
no exchange on the data path (weak scaling).  A batch that one caller owns is
split into contiguous blocks of whole images (image_shard), each rank encodes
its block, and gather_encodings brings the encodings to rank 0 in image order
(strong scaling).  The only collectives are the two
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


def image_shard(offsets, rank: int, world: int):
    """This rank's contiguous block of whole images of a batch (offsets: the
    batch's numImages + 1 row offsets): (first image, end image, the block's
    offsets rebased to its first row).  Blocks differ in size by at most one
    image; a rank may get none."""
    import numpy as np
    n = len(offsets) - 1
    j0, j1 = rank * n // world, (rank + 1) * n // world
    offs = np.asarray(offsets[j0:j1 + 1], dtype=np.int64)
    return j0, j1, offs - offs[0]


def gather_encodings(local, num_images: int, dist):
    """Concatenate every rank's encodings (its image_shard block, rows of a
    2-D tensor) on rank 0 in image order; other ranks receive None.  One
    all-gather of equal-sized, zero-padded blocks."""
    import torch
    if dist is None:
        return local
    world, rank = dist.get_world_size(), dist.get_rank()
    width = local.shape[1]
    most = max((r + 1) * num_images // world - r * num_images // world for r in range(world))
    pad = torch.zeros((most, width), dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad)
    if rank != 0:
        return None
    rows = [parts[r][: (r + 1) * num_images // world - r * num_images // world] for r in range(world)]
    return torch.cat(rows, 0)


def row_shard(n_rows: int, rank: int, world: int) -> tuple[int, int]:
    """This rank's contiguous rows [r0, r1) of n_rows for sharded EM (sizes
    differ by at most one row)."""
    return rank * n_rows // world, (rank + 1) * n_rows // world


def allreduce_sum(dist, group=None):
    """A sum over the ranks of `group` for capi.GMM.em_sharded_device: the
    returned function adds a float64 NumPy array in place over all ranks
    (through a CUDA tensor on an NCCL group, a CPU tensor on gloo)."""
    import numpy as np
    import torch
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"

    def reduce(values: np.ndarray) -> None:
        t = torch.from_numpy(np.ascontiguousarray(values, dtype=np.float64)).to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        values[...] = t.cpu().numpy()
    return reduce
