"""The multi-GPU host logic (vlfeat_b200.replicas) with two gloo ranks on the
CPU: every rank encodes its own data, the step time is the slowest rank's, and
the job's work is the sum of the ranks' descriptors; a batch split into blocks
of whole images, encoded rank by rank (the C restatement standing in for the
GPU on these CPU ranks) and gathered on rank 0, equals the single-process
encoding of the whole batch."""
import multiprocessing as mp
import os
import socket


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, ms, units, out):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from vlfeat_b200 import replicas
        rate, step_ms = replicas.whole_job_rate(units[rank], ms[rank], dist)
        out.put((rank, rate, step_ms, replicas.rank_data_seed(rank)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    ms, units = [4.0, 5.0], [1000.0, 1200.0]
    procs = [ctx.Process(target=_worker, args=(r, 2, port, ms, units, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1]
    for _, rate, step_ms, _ in res:
        assert step_ms == 5.0                      # the slowest rank
        assert abs(rate - 2200.0 / 5e-3) < 1e-6    # all ranks' work over that time
    assert res[0][3] != res[1][3]                  # each replica has its own data


def test_single_process_without_group():
    from vlfeat_b200 import replicas
    assert replicas.whole_job_rate(500.0, 2.0, None) == (250000.0, 2.0)


def _shard_worker(rank, world, port, out):
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle.oracle import FLAG_IMPROVED, Restatement
        from vlfeat_b200 import replicas
        from vlfeat_b200 import workloads as W
        offs, x, (pr, mu, cv) = _batch()
        j0, j1, local = replicas.image_shard(offs, rank, world)
        R = Restatement()
        rows = x[offs[j0]:offs[j1]]
        enc = np.zeros((j1 - j0, 2 * 16 * 8), np.float32)
        for j in range(j1 - j0):
            enc[j] = R.fisher(rows[local[j]:local[j + 1]], mu, cv, pr, FLAG_IMPROVED)[0]
        allenc = replicas.gather_encodings(torch.from_numpy(enc), len(offs) - 1, dist)
        out.put((rank, None if allenc is None else allenc.numpy(), (j0, j1)))
    finally:
        dist.destroy_process_group()


def _batch():
    import numpy as np
    from vlfeat_b200 import workloads as W
    counts = np.array([5, 0, 130, 17, 1, 64, 300])
    offs = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    x = W.pca_like(int(offs[-1]), 8, seed=77)
    return offs, x, W.fv_gmm(16, 8, seed=78)


def test_sharded_batch_gathers_to_single_process_result():
    import numpy as np
    from oracle.oracle import FLAG_IMPROVED, Restatement
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((out.get(timeout=120) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    offs, x, (pr, mu, cv) = _batch()
    assert res[0][2] == (0, 3) and res[1][2] == (3, 7)
    assert res[1][1] is None
    R = Restatement()
    want = np.stack([R.fisher(x[offs[j]:offs[j + 1]], mu, cv, pr, FLAG_IMPROVED)[0] for j in range(len(offs) - 1)])
    assert np.array_equal(res[0][1], want)


def test_image_shard_blocks():
    from vlfeat_b200 import replicas
    offs = [0, 3, 3, 10, 11]
    blocks = [replicas.image_shard(offs, r, 3) for r in range(3)]
    assert [(b[0], b[1]) for b in blocks] == [(0, 1), (1, 2), (2, 4)]
    assert list(blocks[2][2]) == [0, 7, 8]


def _allreduce_worker(rank, world, port, out):
    import datetime

    import numpy as np
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from vlfeat_b200 import replicas
        reduce = replicas.allreduce_sum(dist)
        r0, r1 = replicas.row_shard(1001, rank, world)
        # The sums sharded EM completes: a log-likelihood, then (2D+1)K M-step sums.
        vals = np.arange(r0, r1, dtype=np.float64)
        ll = np.array([vals.sum()])
        reduce(ll)
        stats = np.full(7, float(rank + 1))
        reduce(stats)
        out.put((rank, r0, r1, float(ll[0]), stats.tolist()))
    finally:
        dist.destroy_process_group()


def test_sharded_em_sums_over_two_ranks():
    """The host side of sharded EM on two gloo ranks: row_shard cuts the rows
    into contiguous blocks covering all of them, and allreduce_sum (the
    library's all-reduce callback) sums a float64 array in place on every
    rank."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_allreduce_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, a0, a1, ll0, s0), (_, b0, b1, ll1, s1) = res
    assert (a0, a1, b0, b1) == (0, 500, 500, 1001)
    assert ll0 == ll1 == float(sum(range(1001)))
    assert s0 == s1 == [3.0] * 7
