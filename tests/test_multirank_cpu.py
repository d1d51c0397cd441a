"""Multi-rank host logic on CPU with two gloo ranks (127.0.0.1):
- the bench's replicas: the max of each rank's time over the ranks, then a barrier, agreed by
  every rank, and the job's rate;
- the shot-sharded JointRecon's collectives: the shot partition, the rank-summed normal
  operator, the CG stopping vote, and the LM accept / gather / mean removal, which must give
  exactly what one rank holding every shot computes."""
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


def test_shot_ranges_partition_the_shots():
    from motionest.sharded import shot_range
    for nshots in (4, 7, 64):
        for world in (1, 2, 3, 4):
            if world > nshots:
                continue
            spans = [shot_range(nshots, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == nshots
            assert all(a[1] == b[0] and a[0] < a[1] for a, b in zip(spans, spans[1:]))


def _lm_case(S=7, seed=3):
    import torch
    g = torch.Generator().manual_seed(seed)
    t = torch.randn(S, 6, generator=g, dtype=torch.float64)
    t_next = t + 1e-3 * torch.randn(S, 6, generator=g, dtype=torch.float64)
    t_next[2] = t[2] + 1e-8  # a converged proposal
    stats = torch.rand(S, 28, generator=g, dtype=torch.float64)
    e1 = stats[:, 0] + torch.where(torch.arange(S) % 3 == 0, 0.1, -0.1).to(torch.float64)
    damp = torch.rand(S, generator=g, dtype=torch.float64) + 1e-5
    flags = torch.zeros(S, dtype=torch.uint8)
    return stats, e1, t, t_next, damp, flags


def _sharded_rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from motionest.sharded import (TorchComm, _ReducedProblem, agree_any, lm_accept_gather,
                                       shot_range)
        comm = TorchComm()
        # the CG stopping vote: one rank's pass stops every rank; no pass stops none
        votes = (agree_any(comm, rank == 0, "cpu"), agree_any(comm, False, "cpu"),
                 agree_any(comm, True, "cpu"))
        stats, e1, t, t_next, damp, flags = _lm_case()
        lo, hi = shot_range(t.shape[0], rank, world)
        mean = lm_accept_gather(comm, stats[lo:hi], e1[lo:hi], t, t_next[lo:hi], lo, hi, damp,
                                flags, 1e-6)

        class Fake:  # a rank's partial normal operator: (rank + 1) * p
            def normal(self, p, out):
                out.copy_(p * (rank + 1))
                return out

            def rhs(self, out):
                out.fill_(rank + 1)
                return out

            def residual(self, x, out, energies=None):  # b - A x = (rank + 1) (1 - x)
                out.copy_((1 - x) * (rank + 1))
                if energies is not None:
                    energies.fill_(10.0 * (rank + 1))
                return out

        red = _ReducedProblem(Fake(), comm)
        p = torch.arange(6, dtype=torch.float32).to(torch.complex64) * (1 + 2j)
        ap = red.normal(p, torch.empty_like(p))
        b = red.rhs(torch.empty(3, dtype=torch.complex64))
        en = torch.zeros(2, dtype=torch.float64)
        res = red.residual(p, torch.empty_like(p), energies=en)
        q.put((rank, t.numpy(), damp.numpy(), flags.numpy(), mean.numpy(), ap.numpy(), b.numpy(),
               votes, res.numpy(), en.numpy()))
    finally:
        dist.destroy_process_group()


def test_sharded_collectives_match_one_rank_with_every_shot():
    import multiprocessing as mp
    import numpy as np
    from motionest.sharded import SoloComm, lm_accept_gather
    stats, e1, t, t_next, damp, flags = _lm_case()
    S = t.shape[0]
    mean1 = lm_accept_gather(SoloComm(), stats, e1, t, t_next, 0, S, damp, flags, 1e-6)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict((r, rest) for r, *rest in (q.get(timeout=120) for _ in range(2)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    pp = np.arange(6) * (1 + 2j)
    for r in range(2):
        tr, dr, fr, mr, ap, b, votes, res, en = out[r]
        assert votes == (True, False, True)
        np.testing.assert_array_equal(tr, t.numpy())
        np.testing.assert_array_equal(dr, damp.numpy())
        np.testing.assert_array_equal(fr, flags.numpy())
        np.testing.assert_array_equal(mr, mean1.numpy())
        np.testing.assert_allclose(ap, 3 * pp)  # (1 + 2) p summed over the ranks
        np.testing.assert_allclose(b, 3.0)
        # the initial residual is summed over the ranks (one all-reduce); energies stay local
        np.testing.assert_allclose(res, 3 * (1 - pp))
        np.testing.assert_array_equal(en, 10.0 * (r + 1))
    assert flags[2] == 1 and flags.sum() == 1  # the converged, accepted proposal only
