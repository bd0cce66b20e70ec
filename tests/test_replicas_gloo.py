"""Multi-process replica path of bench.py on CPU: two gloo ranks, each with
its own step times, agree on the slowest rank's times and the whole-job
rate (the GPU runs use the same functions over NCCL)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        times = [100.0 + 10.0 * rank, 50.0 - 5.0 * rank]  # total ms, e2e ms on this rank
        slow = bench.max_over_ranks(times, dist, "cpu")
        dist.barrier()
        q.put((rank, slow, bench.job_rate(world, 20, slow[0])))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for _, slow, rate in res:
        assert slow == [110.0, 50.0]
        assert rate == pytest.approx(2 * 20 / 0.110)
