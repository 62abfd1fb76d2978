"""Host logic of the multi-GPU bench path (one independent replica per rank, no data-path
collective): the job time is the maximum over ranks and the throughput counts every
replica's work.  Two gloo ranks on CPU."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        times = [1.0 + rank, 0.5 * (rank + 1), 2.0 - rank]
        mx = bench.max_over_ranks(dist, times, "cpu")
        v = bench.job_throughput(world, 3e9, mx[0])
        q.put((rank, mx, v))
    finally:
        dist.destroy_process_group()


def test_two_replicas_max_time_and_job_throughput():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, mx, v in res:
        assert mx == pytest.approx([2.0, 1.0, 2.0])
        assert v == pytest.approx(2 * 3e9 / 2.0 / 1e9)
