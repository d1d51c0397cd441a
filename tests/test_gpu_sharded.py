"""Shot-sharded JointRecon on the CUDA kernels, against the single-process JointRecon.

One GPU is available here, so the two ranks run as two host threads on it, each with its own
SENSE problem over its block of shots, exchanging through a host-side all-reduce (a barrier and
a sum in rank order).  No kernel waits on another: the threads only wait for each other on the
host, between launches."""
import threading

import numpy as np
import pytest
import torch

from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu


class _Shared:
    def __init__(self, world):
        self.barrier = threading.Barrier(world, timeout=120)
        self.bufs = [None] * world


class ThreadComm:
    """A communicator for ranks that are threads of one process on one GPU."""

    def __init__(self, rank, world, shared):
        self.rank, self.world, self._s = rank, world, shared

    def all_reduce(self, t):
        torch.cuda.synchronize()
        self._s.bufs[self.rank] = t.clone()
        torch.cuda.synchronize()
        self._s.barrier.wait()
        total = self._s.bufs[0].clone()
        for r in range(1, self.world):
            total += self._s.bufs[r]
        torch.cuda.synchronize()
        self._s.barrier.wait()
        t.copy_(total)
        return t


def _run_ranks(world, make):
    shared = _Shared(world)
    results, errors = [None] * world, []

    def body(r):
        try:
            results[r] = make(ThreadComm(r, world, shared))
        except BaseException as e:  # noqa: BLE001 - reported below
            errors.append(e)
            shared.barrier.abort()

    threads = [threading.Thread(target=body, args=(r,)) for r in range(world)]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=600)
    if errors:
        raise errors[0]
    return results


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_joint_recon_matches_single_process(world):
    from motionest.joint_recon import JointRecon
    from motionest.sharded import ShardedJointRecon
    from motionest.utils import compute_transform_grids_voxel
    d = dict(load_golden("joint"))  # read every array now: the rank threads share them
    kg, rk = compute_transform_grids_voxel(d["ksp"].shape[1:], [1, 1, 1])
    ref = JointRecon(d["ksp"], d["mps"], d["mask"], kg, rk, max_cg_iter=3, max_joint_iter=2)
    xr, tr = ref.run()

    def make(comm):
        app = ShardedJointRecon(d["ksp"], d["mps"], d["mask"], kg, rk, max_cg_iter=3,
                                max_joint_iter=2, comm=comm)
        x, t = app.run()
        torch.cuda.synchronize()
        return x.cpu().numpy(), t.cpu().numpy(), app.objective_history, app.cg_iterations

    out = _run_ranks(world, make)
    for x, t, oh, cgi in out:
        # the shots' partial sums meet in another order than one process adds them: rounding
        np.testing.assert_array_equal(x, out[0][0])  # every rank holds the same image
        assert rel_l2(x, xr.cpu().numpy()) < 1e-5
        np.testing.assert_allclose(t, tr.cpu().numpy(), atol=1e-6)
        np.testing.assert_allclose(oh, ref.objective_history, rtol=1e-5)
        assert cgi == ref.cg_iterations


def test_sharded_single_rank_is_bit_identical_to_joint_recon():
    """One rank holding every shot runs the same kernels, sums the shots' transforms in the same
    order for the mean, and so reproduces JointRecon exactly."""
    from motionest.joint_recon import JointRecon
    from motionest.sharded import ShardedJointRecon, SoloComm
    from motionest.utils import compute_transform_grids_voxel
    d = dict(load_golden("joint"))  # read every array now: the rank threads share them
    kg, rk = compute_transform_grids_voxel(d["ksp"].shape[1:], [1, 1, 1])
    ref = JointRecon(d["ksp"], d["mps"], d["mask"], kg, rk, max_cg_iter=3, max_joint_iter=3)
    xr, tr = ref.run()
    app = ShardedJointRecon(d["ksp"], d["mps"], d["mask"], kg, rk, max_cg_iter=3,
                            max_joint_iter=3, comm=SoloComm())
    x, t = app.run()
    np.testing.assert_array_equal(x.cpu().numpy(), xr.cpu().numpy())
    np.testing.assert_array_equal(t.cpu().numpy(), tr.cpu().numpy())
    np.testing.assert_array_equal(app.damp.cpu().numpy(), ref.damp.cpu().numpy())
    np.testing.assert_array_equal(app.objective_history, ref.objective_history)
