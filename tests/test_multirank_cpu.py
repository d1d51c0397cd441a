"""The multi-GPU bench path on CPU: two gloo ranks (127.0.0.1) run the same collective steps the
bench's replicas take (the max of each rank's time over the ranks, then a barrier) and must agree
on the job's time and rate.  The path is one reconstruction per GPU, so these reductions of the
timing are its only collectives."""
import os
import socket
from datetime import timedelta

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import bench
        ms = bench.rank_max(times[rank], "cpu")
        dist.barrier()
        ms_plain = bench.rank_max(times[rank] * 1.5, "cpu")
        q.put((rank, ms, bench.whole_job_rate(world, 4, ms), ms_plain))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_ranks_agree_on_the_slowest_time_and_the_job_rate(world):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    times = [2900.0, 3100.0]
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, times, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, ms, rate, ms_plain = q.get(timeout=120)
        out[r] = (ms, rate, ms_plain)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        ms, rate, ms_plain = out[r]
        assert ms == max(times)
        assert ms_plain == 1.5 * max(times)
        assert rate == pytest.approx(world * 4 / (max(times) / 1000.0))


def test_single_process_needs_no_group():
    import bench
    assert bench.rank_max(12.5, "cpu") == 12.5
    assert bench.whole_job_rate(1, 4, 2000.0) == pytest.approx(2.0)
