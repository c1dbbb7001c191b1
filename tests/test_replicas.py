"""The multi-GPU host logic of the benchmark (vlfeat_b200.replicas) with two
gloo ranks on the CPU: every rank encodes its own data, the step time is the
slowest rank's, and the job's work is the sum of the ranks' descriptors."""
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
